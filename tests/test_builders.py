"""Native builders (b40c_build_*) against the reference builders' topology."""
import os

import numpy as np
import pytest

import oracle
from back40computing_b200 import (CsrGraph, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph, BuildRandomGraph,
                                  BuildRandomRegularishGraph, sample_sources)


def test_grid_edge_counts_closed_form():
    # grid2d.cuh:63-67, grid3d.cuh:63-68
    for w in (2, 3, 10, 1000):
        g = CsrGraph()
        BuildGrid2dGraph(w, g)
        interior, edge, corner = (w - 2) ** 2, (w - 2) * 4, 4
        assert g.edges == interior * 4 + edge * 3 + corner * 2 + w * w
    for w in (2, 5, 256):
        if w == 256:
            continue  # large case covered by the GPU tests' build
        g = CsrGraph()
        BuildGrid3dGraph(w, g)
        assert g.edges == (w - 2) ** 3 * 6 + (w - 2) ** 2 * 6 * 5 + (w - 2) * 12 * 4 + 8 * 3 + w ** 3


def test_grids_match_golden_topology(golden):
    for name, w, fn in (("grid2d_16", 16, BuildGrid2dGraph), ("grid3d_8", 8, BuildGrid3dGraph),
                        ("grid2d_1", 1, BuildGrid2dGraph)):
        g = CsrGraph()
        fn(w, g)
        assert np.array_equal(g.row_offsets, golden[name]["row_offsets"])
        assert np.array_equal(g.column_indices, golden[name]["column_indices"])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built")
@pytest.mark.parametrize("w", [1, 2, 7, 40])
def test_grids_match_reference_builders(w):
    for kind, fn in (("grid2d", BuildGrid2dGraph), ("grid3d", BuildGrid3dGraph)):
        g = CsrGraph()
        fn(w, g)
        ro, ci = oracle.ref_build(kind, w)
        assert np.array_equal(g.row_offsets, ro) and np.array_equal(g.column_indices, ci)


def _edges_sorted(ro, ci):
    rows = np.repeat(np.arange(ro.size - 1, dtype=np.int64), np.diff(ro))
    key = rows * (ro.size) + ci
    return np.sort(key)


def test_rmat_structure_and_determinism(monkeypatch):
    g1, g2 = CsrGraph(), CsrGraph()
    BuildRmatGraph(1 << 12, 1 << 15, g1, True, 0.57, 0.19, 0.19, seed=3, permute=False)
    monkeypatch.setenv("B40C_BUILD_THREADS", "1")
    BuildRmatGraph(1 << 12, 1 << 15, g2, True, 0.57, 0.19, 0.19, seed=3, permute=False)
    assert np.array_equal(g1.row_offsets, g2.row_offsets)
    assert np.array_equal(g1.column_indices, g2.column_indices)
    assert g1.edges == 2 << 15
    # symmetric multigraph: the sorted (u,v) and (v,u) edge multisets agree
    ro, ci = g1.row_offsets, g1.column_indices
    rows = np.repeat(np.arange(g1.nodes), np.diff(ro))
    fwd = np.sort(rows.astype(np.int64) * g1.nodes + ci)
    rev = np.sort(ci.astype(np.int64) * g1.nodes + rows)
    assert np.array_equal(fwd, rev)
    # the walk starts at (1, 1): without permutation vertex 0 is isolated
    # unless an id wrapped, and the degree distribution is skewed
    deg = np.diff(ro)
    assert deg.max() > 20 * deg.mean()
    g3 = CsrGraph()
    BuildRmatGraph(1 << 12, 1 << 15, g3, True, 0.57, 0.19, 0.19, seed=3, permute=True)
    assert sorted(np.diff(g3.row_offsets)) == sorted(deg)


def test_rmat_degree_profile_close_to_reference():
    """Same generator steps as rmat.cuh (different random stream): the degree
    profile of the seeded builder matches the reference's within sampling noise."""
    if not oracle.have_ref():
        pytest.skip("reference harness not built")
    ro, ci = oracle.ref_build("rmat", 1 << 12, 1 << 15, 1, 0.57, 0.19, 0.19, 0)
    g = CsrGraph()
    BuildRmatGraph(1 << 12, 1 << 15, g, True, 0.57, 0.19, 0.19, seed=0)
    a, b = np.sort(np.diff(ro))[::-1], np.sort(np.diff(g.row_offsets))[::-1]
    assert abs(int((a == 0).sum()) - int((b == 0).sum())) < 0.05 * a.size
    assert 0.7 < b[:50].sum() / a[:50].sum() < 1.3


def test_random_and_rr():
    g = CsrGraph()
    BuildRandomGraph(5000, 20000, g, True, seed=1)
    assert g.edges == 40000 and g.column_indices.min() >= 0 and g.column_indices.max() < 5000
    g = CsrGraph()
    BuildRandomRegularishGraph(4096, 16, g, seed=0)
    assert np.all(np.diff(g.row_offsets) == 16)
    s = CsrGraph()
    BuildRandomRegularishGraph(4096, 16, s, seed=0, symmetrize=True)
    assert s.edges == 2 * 4096 * 16
    # each row starts with its 16 drawn out-neighbours, in draw order (stable by-row CSR)
    for v in (0, 17, 4095):
        assert np.array_equal(s.column_indices[s.row_offsets[v]:s.row_offsets[v] + 16],
                              g.column_indices[g.row_offsets[v]:g.row_offsets[v + 1]])


def test_from_coo_is_stable_by_row():
    rows = np.array([3, 1, 3, 0, 1, 3], np.int32)
    cols = np.array([9, 8, 7, 6, 5, 4], np.int32)
    g = CsrGraph()
    g.FromCoo(rows, cols, 10)
    assert list(g.row_offsets[:5]) == [0, 1, 3, 3, 6]
    assert list(g.column_indices) == [6, 8, 5, 9, 7, 4]


def test_sample_sources_nonzero_degree():
    g = CsrGraph()
    BuildRmatGraph(1 << 12, 1 << 14, g, True, 0.57, 0.19, 0.19, seed=0, permute=True)
    s = sample_sources(g, 64, seed=0)
    assert len(set(s.tolist())) == 64
    assert np.all(np.diff(g.row_offsets)[s] > 0)
    assert np.array_equal(s, sample_sources(g, 64, seed=0))
