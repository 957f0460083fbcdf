"""COO -> CSR on the GPU (b40c_coo_to_csr_device) against the host
conversion, which keeps each row in input order like CsrGraph::FromCoo."""
import ctypes as C

import numpy as np
import pytest

import oracle
from back40computing_b200 import CsrProblem, search, B40cError, DIRECTION_OPTIMIZING
from back40computing_b200 import _native as N

pytestmark = pytest.mark.gpu


def _host_csr(n, rows, cols):
    order = np.argsort(rows, kind="stable")
    ro = np.zeros(n + 1, np.int64)
    np.add.at(ro, rows.astype(np.int64) + 1, 1)
    return np.cumsum(ro).astype(np.int32), cols[order].astype(np.int32)


def _device(n, rows, cols):
    import torch
    d_r = torch.from_numpy(rows.astype(np.int32)).cuda()
    d_c = torch.from_numpy(cols.astype(np.int32)).cuda()
    d_ro = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    d_ci = torch.empty(max(rows.size, 1), dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    rc = N.lib().b40c_coo_to_csr_device(C.c_void_p(d_r.data_ptr()), C.c_void_p(d_c.data_ptr()), n, rows.size,
                                        C.c_void_p(d_ro.data_ptr()), C.c_void_p(d_ci.data_ptr()),
                                        C.c_void_p(s.cuda_stream))
    return rc, d_ro.cpu().numpy(), d_ci.cpu().numpy()[:rows.size]


@pytest.mark.parametrize("n,m", [(1, 0), (1, 5), (200, 5000), (1 << 12, 1 << 16), (1 << 20, 1 << 22),
                                 (1 << 25, 1 << 20), ((1 << 24) + 3, 3 * (1 << 20) + 17)])
def test_matches_stable_host_conversion(n, m):
    rng = np.random.default_rng(n + m)
    # skewed rows (many duplicates) so runs cross tiles and passes
    rows = (rng.pareto(1.5, m) * n / 50).astype(np.int64) % n
    cols = rng.integers(0, n, m)
    rc, ro, ci = _device(n, rows, cols)
    assert rc == 0
    want_ro, want_ci = _host_csr(n, rows, cols)
    assert np.array_equal(ro, want_ro)
    assert np.array_equal(ci, want_ci)


def test_rejects_ids_out_of_range():
    rows = np.array([0, 1, 5], np.int32)
    cols = np.array([1, 2, 0], np.int32)
    rc, _, _ = _device(5, rows, cols)
    assert rc == N.ERROR_INVALID_VALUE


def test_problem_from_coo_searches_like_oracle():
    from back40computing_b200 import CsrGraph, BuildRmatGraph
    g = CsrGraph()
    BuildRmatGraph(1 << 14, 1 << 17, g, True, 0.57, 0.19, 0.19, seed=2, permute=True)
    rows = np.repeat(np.arange(g.nodes, dtype=np.int32), np.diff(g.row_offsets))
    perm = np.random.default_rng(0).permutation(rows.size)
    r, c = rows[perm], g.column_indices[perm]
    p = CsrProblem.from_coo(r, c, g.nodes)
    want_ro, want_ci = _host_csr(g.nodes, r, c)
    for s in (0, 17, 4242):
        got = search(p, s, strategy=DIRECTION_OPTIMIZING)
        want, _ = oracle.bfs(want_ro, want_ci, s)
        assert oracle.compare_labels(got, want) == -1
    with pytest.raises(B40cError):
        CsrProblem.from_coo(np.array([0, 3]), np.array([1, 1]), 3)
