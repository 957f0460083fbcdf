"""The search entry point that allocates nothing (b40c_bfs_search_noalloc).

It serves callers that cannot allocate device memory while they search (a
foreign memory pool, a fixed budget, a stall-free path): they hand in device
pointers for the CSR and the labels and the library supplies the rest from a
fixed scratch array.  This file is collected last so that a run stopping at
its first failure has already run everything else; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from back40computing_b200 import CsrGraph, CsrProblem, BuildRmatGraph, BuildGrid2dGraph, search, sample_sources
from back40computing_b200 import _native as N

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch
    ro = torch.from_numpy(np.ascontiguousarray(g.row_offsets)).cuda()
    ci = torch.from_numpy(np.ascontiguousarray(g.column_indices)).cuda()
    labels = torch.full((g.nodes,), 7, dtype=torch.int32, device="cuda")
    return ro, ci, labels


def _noalloc(ro, ci, g, src, labels):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return N.lib().b40c_bfs_search_noalloc(C.c_void_p(ro.data_ptr()), C.c_void_p(ci.data_ptr()), g.nodes, g.edges,
                                           int(src), C.c_void_p(labels.data_ptr()), C.c_void_p(stream))


@pytest.mark.parametrize("kind", ["rmat", "grid2d", "rmat_at_limits"])
def test_noalloc_matches_expand_contract_twice(kind):
    g = CsrGraph()
    if kind == "rmat":
        BuildRmatGraph(1 << 16, 1 << 20, g, True, 0.57, 0.19, 0.19, seed=4, permute=True)
    elif kind == "rmat_at_limits":
        # 262,144 vertices and 4,194,302 edges: the largest graph the scratch
        # takes (a level's chunk index may then span almost all of its entries)
        BuildRmatGraph(1 << 18, (1 << 21) - 1, g, True, 0.57, 0.19, 0.19, seed=4, permute=True)
        assert g.nodes == 1 << 18 and g.edges == (1 << 22) - 2
    else:
        BuildGrid2dGraph(300, g)
    problem = CsrProblem.from_graph(g)
    ro, ci, labels = _device_csr(g)
    srcs = sample_sources(g, 2, seed=8)
    # two calls in a row: the second starts from the scratch the first left behind
    for s in srcs:
        N.check(_noalloc(ro, ci, g, s, labels), "b40c_bfs_search_noalloc")
        want = search(problem, int(s))  # the allocating entry point, expand-contract distances
        got = labels.cpu().numpy()
        assert np.array_equal(got, want), f"source {s}: first mismatch at {int(np.flatnonzero(got != want)[0])}"


def test_noalloc_rejects_graphs_beyond_its_scratch():
    g = CsrGraph()
    BuildGrid2dGraph(600, g)  # 360,000 vertices > 262,144
    ro, ci, labels = _device_csr(g)
    rc = _noalloc(ro, ci, g, 0, labels)
    assert rc == N.ERROR_INVALID_VALUE
    assert "exceeds its fixed scratch" in N.lib().b40c_last_error_string().decode()


def test_noalloc_labels_at_an_unaligned_address():
    """A caller's labels array need not be 16-byte aligned: the reset falls back
    to 4-byte stores and the neighbouring words stay untouched."""
    import torch
    g = CsrGraph()
    BuildGrid2dGraph(97, g)  # 9,409 vertices: not a multiple of 4
    ro, ci, _ = _device_csr(g)
    buf = torch.full((g.nodes + 2,), 7, dtype=torch.int32, device="cuda")
    labels = buf[1:1 + g.nodes]  # 4 bytes past a 256-byte aligned allocation
    assert labels.data_ptr() % 16 == 4
    N.check(_noalloc(ro, ci, g, 5, labels), "b40c_bfs_search_noalloc")
    y, x = np.divmod(np.arange(g.nodes), 97)
    want = np.abs(x - 5) + y  # L1 distance from vertex 5 on row 0
    got = buf.cpu().numpy()
    assert got[0] == 7 and got[-1] == 7
    assert np.array_equal(got[1:-1], want.astype(np.int32))
