"""Parity of the CUDA BFS path (through the C ABI) with the CPU oracle."""
import numpy as np
import pytest

import oracle
from back40computing_b200 import (CsrGraph, CsrProblem, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph,
                                  BuildRandomRegularishGraph, BuildRandomGraph, search, sample_sources, B40cError)
from back40computing_b200 import _native as N
from back40computing_b200.bfs import EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING, ENACTORS

pytestmark = pytest.mark.gpu

MODES = [N.ENACT_FUSED, N.ENACT_ITERATIVE, N.ENACT_GRAPH]


def _graph(kind, *args, **kw):
    g = CsrGraph()
    if kind == "grid2d":
        BuildGrid2dGraph(args[0], g)
    elif kind == "grid3d":
        BuildGrid3dGraph(args[0], g)
    elif kind == "rmat":
        BuildRmatGraph(args[0], args[1], g, True, 0.57, 0.19, 0.19, seed=kw.get("seed", 0),
                       permute=kw.get("permute", True))
    elif kind == "rr":
        BuildRandomRegularishGraph(args[0], args[1], g, seed=kw.get("seed", 0), symmetrize=kw.get("sym", True))
    elif kind == "random":
        BuildRandomGraph(args[0], args[1], g, kw.get("undirected", True), seed=kw.get("seed", 0))
    return g


def _check_dist(g, problem, src, strategy, mode, **kw):
    got = search(problem, int(src), strategy=strategy, mode=mode, **kw)
    want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(src), kw.get("depth_limit", -1))
    bad = oracle.compare_labels(got, want)
    assert bad == -1, f"label mismatch at {bad}: got {got[bad]} want {want[bad]}"
    return depth


STRATS = [EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID, DIRECTION_OPTIMIZING]


@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("mode", MODES)
def test_golden_fixtures(golden, strategy, mode):
    for name, c in golden.items():
        g = CsrGraph.from_arrays(c["row_offsets"], c["column_indices"])
        p = CsrProblem.from_graph(g)
        for k, s in enumerate(c["sources"]):
            got = search(p, int(s), strategy=strategy, mode=mode)
            assert oracle.compare_labels(got, c[f"labels{k}"]) == -1, name
            enactor = ENACTORS[strategy]()
            enactor._problem = p
            _, depth, _ = enactor.GetStatistics()
            assert depth == int(c[f"depth{k}"]), name


@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind,args", [
    ("grid2d", (100,)), ("grid3d", (20,)), ("rmat", (1 << 14, 1 << 18)), ("rr", (1 << 14, 8)),
    ("random", (20000, 60000)),
])
def test_distance_parity(kind, args, strategy, mode):
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g)
    srcs = sample_sources(g, 3, seed=7)
    for s in srcs:
        _check_dist(g, p, s, strategy, mode)


@pytest.mark.parametrize("strategy", STRATS)
def test_predecessors_valid(strategy):
    g = _graph("rmat", 1 << 14, 1 << 18)
    p = CsrProblem.from_graph(g, mark_predecessors=True)
    for s in sample_sources(g, 3, seed=1):
        preds = search(p, int(s), strategy=strategy)
        dist, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        assert preds[s] == -2
        assert oracle.check_predecessors(g.row_offsets, g.column_indices, dist, preds) == (-1, 0)
        assert np.array_equal(preds >= 0, dist > 0)


@pytest.mark.parametrize("strategy", STRATS)
def test_grid2d_1000_corner_full_size(strategy):
    g = _graph("grid2d", 1000)
    p = CsrProblem.from_graph(g)
    got = search(p, 0, strategy=strategy)
    y, x = np.divmod(np.arange(1_000_000), 1000)
    assert np.array_equal(got, (y + x).astype(np.int32))


def test_depth_limit():
    g = _graph("grid2d", 64)
    p = CsrProblem.from_graph(g)
    for lim in (0, 1, 5, 200):
        _check_dist(g, p, 0, EXPAND_CONTRACT, N.ENACT_FUSED, depth_limit=lim)


def test_isolated_and_edge_cases():
    # vertex 2 has no edges; vertex 3 only a self-loop; source of degree 0
    ro = np.array([0, 1, 2, 2, 3], np.int32)
    ci = np.array([1, 0, 3], np.int32)
    g = CsrGraph.from_arrays(ro, ci)
    p = CsrProblem.from_graph(g)
    for s in range(4):
        _check_dist(g, p, s, EXPAND_CONTRACT, N.ENACT_FUSED)
    with pytest.raises(B40cError) as e:
        search(p, 9)
    assert e.value.status == N.ERROR_INVALID_VALUE


def test_hub_spanning_many_chunks():
    # star: vertex 0 joined to 100k leaves (both directions): one list spans many chunks
    n = 100_001
    rows = np.concatenate([np.zeros(n - 1, np.int32), np.arange(1, n, dtype=np.int32)])
    cols = np.concatenate([np.arange(1, n, dtype=np.int32), np.zeros(n - 1, np.int32)])
    g = CsrGraph()
    g.FromCoo(rows, cols, n)
    p = CsrProblem.from_graph(g)
    for mode in MODES:
        _check_dist(g, p, 0, EXPAND_CONTRACT, mode)
        _check_dist(g, p, 5, EXPAND_CONTRACT, mode)


def test_queue_overflow_status():
    g = _graph("grid2d", 200)
    p = CsrProblem.from_graph(g)
    with pytest.raises(B40cError) as e:
        search(p, 0, queue_sizing=0.001)
    assert e.value.status == N.ERROR_INVALID_CONFIGURATION


def test_repeated_searches_without_reset():
    g = _graph("rmat", 1 << 12, 1 << 15)
    p = CsrProblem.from_graph(g)
    enactor = ENACTORS[EXPAND_CONTRACT]()
    N.check(p.Reset(enactor.GetFrontierType(), 1.3))
    for s in sample_sources(g, 4, seed=3):
        N.check(enactor.EnactFusedSearch(p, int(s)))
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        assert oracle.compare_labels(p.labels(), want) == -1


def test_symmetry_detection():
    g = _graph("rmat", 1 << 12, 1 << 15)
    assert CsrProblem.from_graph(g).is_symmetric()
    d = CsrGraph()
    BuildRandomRegularishGraph(4096, 8, d, seed=1, symmetrize=False)
    assert not CsrProblem.from_graph(d).is_symmetric()


@pytest.mark.parametrize("mode", MODES)
def test_direction_optimizing_goes_bottom_up_and_matches(mode):
    """On R-MAT the large levels run bottom-up: labels and predecessor trees still
    agree with the oracle, also with alpha/beta forcing bottom-up early and long."""
    g = _graph("rmat", 1 << 16, 1 << 20)
    for pred in (False, True):
        p = CsrProblem.from_graph(g, mark_predecessors=pred)
        for alpha, beta in ((0, 0), (1, 1000), (1000, 1)):
            pol = N.Policy()
            pol.bottom_up_alpha, pol.bottom_up_beta = alpha, beta
            for s in sample_sources(g, 2, seed=5):
                got = search(p, int(s), strategy=DIRECTION_OPTIMIZING, mode=mode, policy=pol)
                dist, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
                if pred:
                    assert oracle.check_predecessors(g.row_offsets, g.column_indices, dist, got) == (-1, 0)
                else:
                    assert oracle.compare_labels(got, dist) == -1


def test_direction_optimizing_directed_graph_falls_back():
    d = CsrGraph()
    BuildRandomRegularishGraph(20000, 6, d, seed=2, symmetrize=False)
    p = CsrProblem.from_graph(d)
    for s in (0, 7):
        _check_dist(d, p, s, DIRECTION_OPTIMIZING, N.ENACT_FUSED)


@pytest.mark.parametrize("qa", [1, 2])
def test_queue_allocation_modes(qa):
    g = _graph("rmat", 1 << 14, 1 << 18)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.queue_allocation = qa
    for strategy in (EXPAND_CONTRACT, TWO_PHASE):
        for s in sample_sources(g, 2, seed=9):
            got = search(p, int(s), strategy=strategy, policy=pol)
            want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            assert oracle.compare_labels(got, want) == -1


@pytest.mark.parametrize("small", [-1, 256, 1 << 30])
@pytest.mark.parametrize("strategy", [EXPAND_CONTRACT, DIRECTION_OPTIMIZING])
def test_small_frontier_path(small, strategy):
    """Runs of small levels on one CTA (or never, or always) give the same labels."""
    pol = N.Policy()
    pol.small_frontier_edges = small
    for kind, args in (("grid2d", (70,)), ("rmat", (1 << 13, 1 << 16)), ("grid3d", (12,))):
        g = _graph(kind, *args)
        p = CsrProblem.from_graph(g)
        for s in sample_sources(g, 2, seed=4):
            got = search(p, int(s), strategy=strategy, policy=pol)
            want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            assert oracle.compare_labels(got, want) == -1


def test_instrumentation_records_levels():
    g = _graph("grid2d", 40)
    p = CsrProblem.from_graph(g)
    p.set_instrument(True)
    got = search(p, 0)
    recs = p.level_records()
    assert len(recs) == int(got.max()) + 2  # one per level plus the empty last frontier
    hist = oracle.level_histogram(got)
    # a level's frontier is the vertices at that distance (all have edges on a lattice)
    assert [r["vertices"] for r in recs[:-1]] == [int(c) for c in hist]
    enactor = ENACTORS[EXPAND_CONTRACT]()
    enactor._problem = p
    _, depth, duty = enactor.GetStatistics()
    assert depth == int(got.max()) + 1 and 0.0 < duty <= 1.0


# ---- batched multi-source searches ------------------------------------------------------

@pytest.mark.parametrize("kind,args", [("rmat", (1 << 14, 1 << 18)), ("rr", (1 << 14, 8)), ("grid2d", (90,)),
                                       ("random", (20000, 60000))])
def test_batched_matches_single_source(kind, args):
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g)
    srcs = sample_sources(g, 64, seed=11)
    p.msbfs(srcs)
    for slot in (0, 1, 17, 63):
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1


def test_batched_depth_limits_duplicates_and_small_batches():
    g = _graph("rmat", 1 << 13, 1 << 17)
    p = CsrProblem.from_graph(g)
    base = sample_sources(g, 5, seed=2)
    srcs = np.array([base[0], base[1], base[0], base[2], base[3], base[1], base[4]], np.int32)  # duplicates
    limits = np.array([-1, 2, 3, 0, -1, -1, 1], np.int32)
    p.msbfs(srcs, limits)
    for slot in range(srcs.size):
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[slot]), int(limits[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1
    p.msbfs(srcs[:1])
    want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[0]))
    assert oracle.compare_labels(p.labels_of(0), want) == -1
    with pytest.raises(B40cError):
        p.labels_of(1)
    with pytest.raises(B40cError):
        p.msbfs(np.zeros(65, np.int32))


def test_batched_directed_graph_push_only():
    d = CsrGraph()
    BuildRandomRegularishGraph(30000, 6, d, seed=3, symmetrize=False)
    p = CsrProblem.from_graph(d)
    srcs = np.arange(0, 64 * 400, 400, dtype=np.int32)
    p.msbfs(srcs)
    for slot in (0, 33, 63):
        want, _ = oracle.bfs(d.row_offsets, d.column_indices, int(srcs[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1


@pytest.mark.parametrize("alpha", [1, 1000])
def test_batched_pull_threshold_extremes(alpha):
    """alpha = 1: only very dense levels pull; alpha = 1000: nearly every level pulls."""
    g = _graph("rmat", 1 << 14, 1 << 18)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.bottom_up_alpha = alpha
    srcs = sample_sources(g, 64, seed=21)
    lim = np.where(np.arange(64) % 5 == 0, 3, -1).astype(np.int32)
    p.msbfs(srcs, lim, policy=pol)
    for slot in (0, 5, 31, 62):
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[slot]), int(lim[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1


def test_batch_then_single_source_on_same_problem():
    g = _graph("rmat", 1 << 13, 1 << 16)
    p = CsrProblem.from_graph(g)
    srcs = sample_sources(g, 8, seed=30)
    p.msbfs(srcs)
    got = search(p, int(srcs[2]), strategy=DIRECTION_OPTIMIZING)
    want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[2]))
    assert oracle.compare_labels(got, want) == -1
    assert oracle.compare_labels(p.labels_of(2), want) == -1


@pytest.mark.parametrize("strategy", [EXPAND_CONTRACT, DIRECTION_OPTIMIZING, CONTRACT_EXPAND])
@pytest.mark.parametrize("mode", [N.ENACT_FUSED, N.ENACT_GRAPH])
def test_queued_enacts_keep_their_sources(strategy, mode):
    """Enacts are asynchronous: three searches queued back to back (a long path
    search, the same long search, then a search from an isolated vertex) must
    each run from their own source, even though the host returns long before
    the GPU reaches the second one."""
    L = 6000
    ro = np.zeros(L + 2, np.int32)
    deg = np.full(L, 2, np.int32)
    deg[0] = deg[-1] = 1
    ro[1:L + 1] = np.cumsum(deg)
    ro[L + 1] = ro[L]
    ci = np.empty(ro[L], np.int32)
    for v in range(L):
        nb = [u for u in (v - 1, v + 1) if 0 <= u < L]
        ci[ro[v]:ro[v] + len(nb)] = nb
    g = CsrGraph.from_arrays(ro, ci)
    p = CsrProblem.from_graph(g)
    e = ENACTORS[strategy]()
    N.check(p.Reset(e.GetFrontierType(), 1.3))
    N.check(e._enact(p, 0, mode, 0))  # warm-up (graph build, symmetry check)
    p.labels()
    for s in (0, 0, L):
        N.check(e._enact(p, s, mode, 0))
    t = p.recent_search_ms(3)
    got = p.labels()
    want = np.full(L + 1, -1, np.int32)
    want[L] = 0
    assert oracle.compare_labels(got, want) == -1
    assert t[1] > 5 * t[2], f"second queued search ran short ({t}): it did not search from its own source"
    assert t[1] > 0.5 * t[0], t


def test_many_queued_enacts_wrap_the_source_ring():
    """More queued enacts than the per-handle ring of source slots (256)."""
    g = _graph("rmat", 1 << 12, 1 << 15)
    p = CsrProblem.from_graph(g)
    e = ENACTORS[DIRECTION_OPTIMIZING]()
    N.check(p.Reset(e.GetFrontierType(), 1.3))
    srcs = sample_sources(g, 7, seed=3)
    for i in range(300):
        N.check(e._enact(p, int(srcs[i % 7]), N.ENACT_FUSED, 0))
    want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[299 % 7]))
    assert oracle.compare_labels(p.labels(), want) == -1


@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("mode", MODES)
def test_source_without_edges(strategy, mode):
    """A source with no edges: an empty first frontier must end the search in
    every mode (in a captured graph the loop condition is set to stop)."""
    g = _graph("rmat", 1 << 12, 1 << 15)
    deg = np.diff(g.row_offsets)
    iso = int(np.flatnonzero(deg == 0)[0])
    p = CsrProblem.from_graph(g)
    for s in (iso, int(sample_sources(g, 1, seed=4)[0]), iso):
        got = search(p, s, strategy=strategy, mode=mode)
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, s)
        assert oracle.compare_labels(got, want) == -1
        e = ENACTORS[strategy]()
        e._problem = p
        assert e.GetStatistics()[1] == depth


@pytest.mark.parametrize("scan,hub,defer", [(1, 1, 1), (1, -1, 1), (1, 1, -1)])
@pytest.mark.parametrize("kind,args", [("rmat", (1 << 15, 1 << 19)), ("rr", (1 << 15, 12)), ("grid3d", (24,))])
@pytest.mark.parametrize("preds", [False, True])
def test_bottom_up_scan_variants(scan, hub, defer, kind, args, preds):
    """Bottom-up levels with and without the hub-pair probes, with the frontier
    deferred (built from the mask buffers when a top-down level follows) or
    emitted, give the oracle's distances and valid predecessors; alpha 2 forces
    many bottom-up levels."""
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g, mark_predecessors=preds)
    pol = N.Policy()
    pol.bottom_up_scan = scan
    pol.bottom_up_hub_probes = hub
    pol.bottom_up_defer_frontier = defer
    pol.bottom_up_alpha = 2
    for s in sample_sources(g, 3, seed=9):
        got = search(p, int(s), strategy=DIRECTION_OPTIMIZING, policy=pol)
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        if preds:
            assert got[s] == -2
            assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
        else:
            assert oracle.compare_labels(got, want) == -1


@pytest.mark.parametrize("hub", [1, -1])
@pytest.mark.parametrize("kind,args", [("rmat", (1 << 15, 1 << 19)), ("rr", (1 << 14, 10))])
def test_batched_pull_hub_probes(hub, kind, args):
    """Batched searches with and without the hub-pair probes in pull levels
    (alpha 2 makes most levels pull) give every slot the oracle's labels."""
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g)
    srcs = sample_sources(g, 40, seed=12)
    pol = N.Policy()
    pol.bottom_up_hub_probes = hub
    pol.bottom_up_alpha = 2
    p.msbfs(srcs, policy=pol)
    depths = p.msbfs_depths()
    for slot in (0, 7, 39):
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1
        assert depths[slot] == depth


@pytest.mark.parametrize("lists,defer", [(1, 1), (-1, 1), (-1, -1)])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("alpha,beta", [(2, 1), (2, 24), (2, 1000), (1, 2)])
@pytest.mark.parametrize("kind,args", [("rmat", (1 << 15, 1 << 19)), ("rr", (1 << 14, 10)), ("grid3d", (20,))])
def test_bottom_up_list_mode_and_alternation(lists, defer, mode, alpha, beta, kind, args):
    """Direction switches in every pattern (bottom-up runs, bottom-up -> top-down
    -> bottom-up with the unvisited list carried over and top-down levels
    claiming on the labels, deferred bottom-up frontiers built before a
    top-down level or a solo phase) give the oracle's distances in every
    launch mode."""
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g)
    pol = N.Policy()
    pol.bottom_up_alpha = alpha
    pol.bottom_up_beta = beta
    pol.bottom_up_list = lists
    pol.bottom_up_defer_frontier = defer
    for s in sample_sources(g, 3, seed=21):
        got = search(p, int(s), strategy=DIRECTION_OPTIMIZING, mode=mode, policy=pol)
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        assert oracle.compare_labels(got, want) == -1
        e = ENACTORS[DIRECTION_OPTIMIZING]()
        e._problem = p
        assert e.GetStatistics()[1] == depth


@pytest.mark.parametrize("preds", [False, True])
def test_pipelined_extract_matches_sync(preds):
    """Read-back through the two staging slots while later searches run gives,
    for every search, the labels the synchronous read-back gives."""
    g = _graph("rmat", 1 << 14, 1 << 18)
    p = CsrProblem.from_graph(g, mark_predecessors=preds)
    e = ENACTORS[DIRECTION_OPTIMIZING]()
    N.check(p.Reset(e.GetFrontierType(), 1.3))
    srcs = [int(s) for s in sample_sources(g, 6, seed=4)]
    bufs = [np.full(g.nodes, 7, np.int32) for _ in range(2)]
    got = {}
    for i, s in enumerate(srcs):
        N.check(e._enact(p, s, N.ENACT_FUSED, 0))
        slot = i & 1
        if i >= 2:  # the slot's previous search: wait, then keep a copy before the buffer is reused
            N.check(p.ExtractWait(slot))
            got[srcs[i - 2]] = bufs[slot].copy()
        N.check(p.ExtractResultsAsync(bufs[slot], slot))
    for i in (len(srcs) - 2, len(srcs) - 1):
        N.check(p.ExtractWait(i & 1))
        got[srcs[i]] = bufs[i & 1].copy()
    assert p.ExtractWait(0) == 0  # nothing in flight: returns at once
    for s in srcs:
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, s)
        if preds:
            assert got[s][s] == -2
            assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got[s]) == (-1, 0)
        else:
            assert oracle.compare_labels(got[s], want) == -1
    with pytest.raises(B40cError):
        N.check(p.ExtractResultsAsync(bufs[0], 2))


@pytest.mark.parametrize("threshold", [4096, 65536])
@pytest.mark.parametrize("kind,args,strategy", [("grid2d", (300,), EXPAND_CONTRACT), ("grid3d", (40,), EXPAND_CONTRACT),
                                                 ("rmat", (1 << 15, 1 << 19), DIRECTION_OPTIMIZING),
                                                 ("rr", (1 << 15, 12), EXPAND_CONTRACT)])
@pytest.mark.parametrize("preds", [False, True])
def test_subgrid_phase(threshold, kind, args, strategy, preds):
    """Runs of mid-size top-down levels on 16 CTAs with their own barrier (the
    sub-grid phase, entered and left level by level between solo phases and
    whole-grid levels) give the oracle's distances, valid predecessors and the
    search depth."""
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g, mark_predecessors=preds)
    pol = N.Policy()
    pol.subgrid_frontier_edges = threshold
    pol.ctas_per_sm = 1  # 148 CTAs: the phase needs at least 64
    srcs = [0] if kind.startswith("grid") else [int(s) for s in sample_sources(g, 2, seed=17)]
    for s in srcs:
        got = search(p, s, strategy=strategy, policy=pol)
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, s)
        if preds:
            assert got[s] == -2
            assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
        else:
            assert oracle.compare_labels(got, want) == -1
            e = ENACTORS[strategy]()
            e._problem = p
            assert e.GetStatistics()[1] == depth


# ---- sources joining a batch in flight ------------------------------------------------

@pytest.mark.parametrize("kind,args", [("grid2d", (400,)), ("rmat", (1 << 16, 1 << 20)), ("rr", (1 << 15, 8))])
def test_sources_join_a_running_batch(kind, args):
    """Sources added while a batch runs (b40c_msbfs_join) are taken at a level
    boundary and searched from there on in their own slots: each joined slot's
    labels and search depth equal the oracle's for that source alone, and the
    batch's own slots are unchanged."""
    import ctypes as C
    g = _graph(kind, *args)
    p = CsrProblem.from_graph(g)
    srcs = sample_sources(g, 12, seed=41)
    p.msbfs(srcs[:16] if srcs.size > 16 else srcs)  # sizes the label rows (12)
    base, joins = srcs[:4], srcs[4:12]
    lim = np.array([-1, 3, -1, 0, -1, 5, -1, -1], np.int32)
    p.msbfs(base)
    for j, s in enumerate(joins):
        p.msbfs_join(4 + j, int(s), int(lim[j]))
    taken, depths = p.msbfs_joined()
    assert 0 <= taken <= joins.size
    for slot in range(4):
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(base[slot]))
        assert oracle.compare_labels(p.labels_of(slot), want) == -1
        assert depths[slot] == depth
    for j in range(taken):
        want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(joins[j]), int(lim[j]))
        assert oracle.compare_labels(p.labels_of(4 + j), want) == -1, f"joined slot {4 + j}"
        assert depths[4 + j] == depth, f"joined slot {4 + j}"
    with pytest.raises(B40cError):
        p.msbfs_join(2, int(joins[0]))  # a slot of the batch's own sources
    with pytest.raises(B40cError):
        p.msbfs_join(12, int(joins[0]))  # past the label rows
    p.Destroy()


def test_join_taken_while_a_long_batch_runs():
    """On a lattice the batch takes thousands of levels: requests sent right
    after the launch are all taken, at different levels, with exact labels."""
    g = _graph("grid2d", 1000)
    p = CsrProblem.from_graph(g)
    p.msbfs(np.arange(0, 8, dtype=np.int32) * 1000)  # label rows for 8 slots
    p.msbfs(np.array([0], np.int32))  # corner: about 2,000 levels
    joins = [999, 500_500, 999_999, 123_456]
    for j, s in enumerate(joins):
        p.msbfs_join(1 + j, s, -1)
    taken, depths = p.msbfs_joined()
    assert taken == len(joins)
    y, x = np.divmod(np.arange(1_000_000), 1000)
    for j, s in enumerate(joins):
        sy, sx = divmod(s, 1000)
        want = (np.abs(x - sx) + np.abs(y - sy)).astype(np.int32)
        assert np.array_equal(p.labels_of(1 + j), want), f"joined source {s}"
        assert depths[1 + j] == int(want.max()) + 1
    p.Destroy()


@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("preds", [False, True])
def test_history_cull(strategy, mode, preds):
    """With the per-CTA history table on, repeats of neighbours already sent to
    the visited test are dropped in shared memory: distances still equal the
    oracle's and predecessors stay valid (R-MAT hubs repeat a lot; the
    lattice's neighbours repeat across levels)."""
    pol = N.Policy()
    pol.history_cull = 1
    for kind, args in (("rmat", (1 << 15, 1 << 19)), ("grid2d", (120,)), ("random", (20000, 60000))):
        g = _graph(kind, *args)
        p = CsrProblem.from_graph(g, mark_predecessors=preds)
        for s in sample_sources(g, 2, seed=13):
            got = search(p, int(s), strategy=strategy, mode=mode, policy=pol)
            want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            if preds:
                assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
            else:
                assert oracle.compare_labels(got, want) == -1, f"{kind} source {s}"
        p.Destroy()


@pytest.mark.parametrize("threads", [128, 256, 512])
@pytest.mark.parametrize("prefetch", [1, -1])
@pytest.mark.parametrize("preds", [False, True])
@pytest.mark.parametrize("warp_bu", [1, -1])
def test_cta_sizes_and_bottom_up_prefetch(threads, prefetch, preds, warp_bu):
    """Every strategy built for 128-, 256- and 512-thread CTAs, and counting
    bottom-up levels warp by warp or in CTA-wide chunks (the first level of a
    run with and without its chunks staged by bulk copies), gives the
    oracle's distances and valid predecessors (graphs whose vertex count is
    not a multiple of the chunk, so the ragged last chunk is covered)."""
    pol = N.Policy()
    pol.threads = threads
    pol.bottom_up_prefetch = prefetch
    pol.warp_bottom_up = warp_bu
    pol.bottom_up_alpha = 4
    for kind, args in (("rmat", (1 << 15, 1 << 19)), ("rr", (20011, 10)), ("grid3d", (23,))):
        g = _graph(kind, *args)
        p = CsrProblem.from_graph(g, mark_predecessors=preds)
        for strategy in (DIRECTION_OPTIMIZING, EXPAND_CONTRACT, CONTRACT_EXPAND):
            for s in sample_sources(g, 2, seed=19):
                got = search(p, int(s), strategy=strategy, policy=pol)
                want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
                if preds:
                    assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
                else:
                    assert oracle.compare_labels(got, want) == -1, f"{kind} {strategy} source {s}"
        if not preds:
            srcs = sample_sources(g, 20, seed=3)
            p.msbfs(srcs, policy=pol)
            for slot in (0, 19):
                want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(srcs[slot]))
                assert oracle.compare_labels(p.labels_of(slot), want) == -1
        p.Destroy()


@pytest.mark.parametrize("warp_contract", [1, -1])
@pytest.mark.parametrize("strategy", [EXPAND_CONTRACT, CONTRACT_EXPAND, TWO_PHASE, HYBRID])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("preds", [False, True])
@pytest.mark.parametrize("grid", [0, 16])
def test_levels_by_warps_and_by_ctas(warp_contract, strategy, mode, preds, grid):
    """Top-down levels of expand-contract and the contract and expand passes
    of the edge-frontier strategies, warp by warp (each warp flushing its own
    winners to the vertex frontier; the default for levels with a full
    sub-round per CTA) or in CTA-wide sub-rounds: the oracle's distances,
    valid predecessors, and the reference's total_queued (expand-contract:
    the reached vertices but the source; the others: the edges of the reached
    vertices).  A 16-CTA grid puts the larger levels of these graphs on the
    warp path.  The R-MAT graph has hubs whose lists span many 256-edge
    chunks (their chunk-index runs are written by the whole warp); the
    directed graph has vertices without out-edges (labelled, never
    enqueued)."""
    pol = N.Policy()
    pol.warp_contract = warp_contract
    for kind, args, kw in (("rmat", (1 << 16, 1 << 20), {}), ("rr", (30011, 5), {"sym": False}),
                           ("grid2d", (150,), {})):
        g = _graph(kind, *args, **kw)
        assert kind != "rmat" or np.diff(g.row_offsets).max() > 8 * 256
        p = CsrProblem.from_graph(g, mark_predecessors=preds)
        e = ENACTORS[strategy](policy=pol)
        e._problem = p
        for s in sample_sources(g, 2, seed=23):
            got = search(p, int(s), strategy=strategy, mode=mode, policy=pol, max_grid_size=grid)
            want, depth = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            if preds:
                assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
            else:
                assert oracle.compare_labels(got, want) == -1, f"{kind} source {s}"
                nv, ev = oracle.visited_stats(g.row_offsets, got)
                queued = nv - 1 if strategy == EXPAND_CONTRACT else ev
                assert e.GetStatistics()[0] == queued, f"{kind} source {s}: total_queued"
        p.Destroy()


@pytest.mark.parametrize("threads", [256, 512])
@pytest.mark.parametrize("preds", [False, True])
@pytest.mark.parametrize("grid", [0, 7])
def test_bottom_up_level_by_warps(threads, preds, grid):
    """The first bottom-up level of a run warp by warp (blocks of vertex ids
    dealt over every warp of the grid, no CTA barriers): the oracle's
    distances and valid predecessors on power-law, uniform and lattice
    graphs, with a low switching threshold so that several bottom-up runs
    occur, on the whole device and on a 7-CTA grid (many blocks per warp)."""
    pol = N.Policy()
    pol.threads = threads
    pol.warp_bottom_up = 1
    pol.bottom_up_alpha = 4
    for kind, args in (("rmat", (1 << 16, 1 << 20)), ("rr", (40009, 8)), ("grid2d", (181,))):
        g = _graph(kind, *args)
        p = CsrProblem.from_graph(g, mark_predecessors=preds)
        for s in sample_sources(g, 3, seed=29):
            got = search(p, int(s), strategy=DIRECTION_OPTIMIZING, policy=pol, max_grid_size=grid)
            want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
            if preds:
                assert oracle.check_predecessors(g.row_offsets, g.column_indices, want, got) == (-1, 0)
            else:
                assert oracle.compare_labels(got, want) == -1, f"{kind} source {s}"
        p.Destroy()
