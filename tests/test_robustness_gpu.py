"""Zero-copy CSR, caller arrays at odd addresses, the search statistics'
definitions, the sub-grid phase, and device-side waits that run out."""
import ctypes as C

import numpy as np
import pytest

import oracle
from back40computing_b200 import (CsrGraph, CsrProblem, BuildGrid3dGraph, BuildRmatGraph,
                                  BuildRandomRegularishGraph, search, sample_sources, B40cError)
from back40computing_b200 import _native as N
from back40computing_b200.bfs import (EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING,
                                      ENACTORS)

pytestmark = pytest.mark.gpu

MODES = [N.ENACT_FUSED, N.ENACT_ITERATIVE, N.ENACT_GRAPH]
STRATS = [EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING]


def _rmat(scale, ef=16, seed=0):
    g = CsrGraph()
    BuildRmatGraph(1 << scale, ef << scale, g, True, 0.57, 0.19, 0.19, seed=seed, permute=True)
    return g


def _at_offset(a, offset_words):
    """A copy of int32 array `a` placed `offset_words` int32 past a 64-byte
    boundary of a larger buffer (the buffer is returned too, to keep it alive)."""
    buf = np.zeros(a.size + 32, np.int32)
    base = (-(buf.ctypes.data // 4)) % 16  # words to the next 64-byte boundary
    view = buf[base + offset_words: base + offset_words + a.size]
    view[:] = a
    assert view.ctypes.data % 64 == 4 * offset_words
    return buf, view


# ---- zero-copy stream-from-host (csr_problem.cuh:351-363) -----------------------------

@pytest.mark.parametrize("offset_words", [0, 1])
@pytest.mark.parametrize("strategy", STRATS)
def test_stream_from_host_matches_oracle(strategy, offset_words):
    """The kernels read the caller's host CSR over the bus (mapped, not
    copied), also when its column array starts 4 bytes past a 16-byte boundary;
    labels equal the oracle's in every launch mode."""
    g = _rmat(15)
    keep_ro, ro = _at_offset(g.row_offsets, offset_words)
    keep_ci, ci = _at_offset(g.column_indices, offset_words)
    p = CsrProblem()
    N.check(p.FromHostProblem(True, g.nodes, g.edges, ci, ro, 1), "FromHostProblem(stream_from_host)")
    assert p.device_view().d_column_indices != 0
    for mode in MODES:
        for s in sample_sources(g, 2, seed=3):
            got = search(p, int(s), strategy=strategy, mode=mode)
            want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            assert oracle.compare_labels(got, want) == -1, f"source {s}, mode {mode}"
    p.Destroy()
    del keep_ro, keep_ci


def test_device_column_array_at_odd_offsets_uses_bulk_staging_correctly():
    """A sub-round inside one long adjacency list is staged into shared memory
    by one bulk copy whose start is rounded to a 16-byte boundary by address:
    the no-allocation search takes the caller's device column array, so place
    it 4, 8 and 12 bytes past a boundary on a graph with long lists."""
    import torch
    g = _rmat(16)
    assert np.diff(g.row_offsets).max() > 4096  # hub lists span whole sub-rounds
    ref = CsrProblem.from_graph(g)
    ro = torch.from_numpy(g.row_offsets).cuda()
    srcs = sample_sources(g, 2, seed=6)
    for off in (1, 2, 3):
        buf = torch.zeros(g.edges + 8, dtype=torch.int32, device="cuda")
        ci = buf[off: off + g.edges]
        ci.copy_(torch.from_numpy(g.column_indices))
        assert ci.data_ptr() % 16 == 4 * off
        labels = torch.full((g.nodes,), 7, dtype=torch.int32, device="cuda")
        for s in srcs:
            N.check(N.lib().b40c_bfs_search_noalloc(C.c_void_p(ro.data_ptr()), C.c_void_p(ci.data_ptr()), g.nodes,
                                                    g.edges, int(s), C.c_void_p(labels.data_ptr()),
                                                    C.c_void_p(torch.cuda.current_stream().cuda_stream)))
            want = search(ref, int(s))
            assert np.array_equal(labels.cpu().numpy(), want), f"offset {4 * off} bytes, source {s}"
    ref.Destroy()


def _directed_with_sinks(n, degree, every):
    """A directed graph of `degree` random out-neighbours per vertex in which
    every `every`-th vertex has no out-edges: such vertices are reached and
    labelled but never expanded."""
    d = CsrGraph()
    BuildRandomRegularishGraph(n, degree, d, seed=5, symmetrize=False)
    ro, ci = d.row_offsets, d.column_indices
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(ro))
    keep = rows % every != 0
    g = CsrGraph()
    g.FromCoo(rows[keep], ci[keep], n)
    return g


# ---- statistics: total_queued (enactor_contract_expand.cuh:237-250) ---------------------

@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("kind", ["rmat", "directed"])
def test_total_queued_matches_the_reference_definition(kind, strategy, mode):
    """The reference sums the queue lengths of every iteration after the
    source's: for the edge-frontier strategies (contract-expand, two-phase,
    hybrid) that is the edges of the reached vertices, for expand-contract the
    reached vertices other than the source (its vertex queue keeps vertices
    without edges too); with exact culling no duplicate adds to either."""
    g = _rmat(14) if kind == "rmat" else _directed_with_sinks(20000, 3, 7)
    p = CsrProblem.from_graph(g)
    for s in sample_sources(g, 3, seed=2):
        got = search(p, int(s), strategy=strategy, mode=mode)
        nv, ev = oracle.visited_stats(g.row_offsets, got)
        e = ENACTORS[strategy]()
        e._problem = p
        total_queued = e.GetStatistics()[0]
        want = nv - 1 if strategy in (EXPAND_CONTRACT, DIRECTION_OPTIMIZING) else ev
        assert total_queued == want, f"source {s}: total_queued {total_queued}, want {want}"


# ---- the sub-grid phase runs --------------------------------------------------------------

def test_subgrid_phase_is_entered():
    """With no solo phase and a sub-grid threshold above every level of a
    lattice, the levels run on the first 16 CTAs alone: in the per-CTA clock
    records only CTAs below 16 start work in those passes, several of them do
    once a level has more than a few hundred edges, and the distances stay
    exact."""
    w = 40
    g = CsrGraph()
    BuildGrid3dGraph(w, g)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.subgrid_frontier_edges = 1 << 20
    pol.small_frontier_edges = -1
    pol.ctas_per_sm = 1  # 148 CTAs: the phase needs at least 64
    p.set_instrument(True)
    got = search(p, 0, policy=pol)
    idx = np.arange(w ** 3)
    assert np.array_equal(got, (idx % w + idx // w % w + idx // (w * w)).astype(np.int32))
    arr = p.cta_arrivals(64, phases=True)  # [pass][cta][phase]
    assert arr.shape[1] >= 64
    started = arr[:, :, 0] > 0  # phase 0: the CTA began a work chunk of the level
    shared = 0
    for k in range(15, 64):     # levels of about 900 to 8,000 edges
        who = np.flatnonzero(started[k])
        assert who.size >= 1 and who.max() < 16, f"pass {k}: CTAs {who[:20]}"
        shared += who.size >= 2
    assert shared >= 40
    p.set_instrument(False)
    p.Destroy()


# ---- device-side waits that run out ----------------------------------------------------

@pytest.mark.parametrize("strategy", [EXPAND_CONTRACT, DIRECTION_OPTIMIZING, CONTRACT_EXPAND, HYBRID])
def test_barrier_wait_runs_out_and_the_problem_stays_usable(monkeypatch, strategy):
    """A CTA that leaves without arriving at the grid barrier (a test-only
    switch; it reports nothing) leaves every other CTA waiting: their waits,
    bounded by a short test-only poll limit, run out, the search returns
    B40C_ERROR_LAUNCH_TIMEOUT (702) instead of hanging, and the next search on
    the same problem gives the oracle's labels."""
    g = _rmat(16)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.small_frontier_edges = -1  # every level on the whole grid
    s = int(sample_sources(g, 1, seed=1)[0])
    want, _ = oracle.bfs(g.row_offsets, g.column_indices, s)
    monkeypatch.setenv("B40C_TEST_SKIP_ARRIVAL_CTA", "3")
    monkeypatch.setenv("B40C_TEST_SPIN_LIMIT", "4096")
    with pytest.raises(B40cError) as e:
        search(p, s, strategy=strategy, policy=pol)
    assert e.value.status == N.ERROR_LAUNCH_TIMEOUT
    monkeypatch.delenv("B40C_TEST_SKIP_ARRIVAL_CTA")
    monkeypatch.delenv("B40C_TEST_SPIN_LIMIT")
    got = search(p, s, strategy=strategy, policy=pol)
    assert oracle.compare_labels(got, want) == -1
    p.Destroy()


# ---- CTAs that start late ------------------------------------------------------------

@pytest.mark.parametrize("strategy", [EXPAND_CONTRACT, DIRECTION_OPTIMIZING, CONTRACT_EXPAND, HYBRID])
@pytest.mark.parametrize("threads", [256, 512])
def test_ctas_that_start_late_join_at_the_first_level(monkeypatch, strategy, threads):
    """Every CTA but CTA 0 of the persistent launch starts 300 us late (a
    test-only switch), long after CTA 0 has finished its share of the first
    level: the late CTAs still start at that level (block 0 advances the level
    only after the end-of-level barrier), so the labels and the search depth
    are the oracle's."""
    g = _rmat(14)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.threads = threads
    pol.small_frontier_edges = -1  # the first level on the whole grid, not CTA 0 alone
    monkeypatch.setenv("B40C_TEST_LATE_START_NS", "300000")
    for s in sample_sources(g, 3, seed=9):
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        got = search(p, int(s), strategy=strategy, policy=pol)
        assert oracle.compare_labels(got, want) == -1
        e = ENACTORS[strategy]()
        e._problem = p
        assert e.GetStatistics()[1] == depth
    p.Destroy()
