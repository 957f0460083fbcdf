"""The query server (include/b40c_server.h) against the oracle: answers in a
mixed, batched stream equal the answers of the same queries searched alone."""
import numpy as np
import pytest

import oracle
from back40computing_b200 import CsrGraph, CsrProblem, BuildGrid2dGraph, BuildRmatGraph, BuildRandomGraph
from back40computing_b200 import BuildRandomRegularishGraph, sample_sources, search, B40cError
from back40computing_b200 import _native as N
from back40computing_b200.server import BfsServer, latency_summary

pytestmark = pytest.mark.gpu


def _graphs():
    gs = []
    g = CsrGraph()
    BuildRmatGraph(1 << 13, 1 << 16, g, True, 0.57, 0.19, 0.19, seed=3, permute=True)
    gs.append(g)
    g = CsrGraph()
    BuildGrid2dGraph(90, g)
    gs.append(g)
    g = CsrGraph()
    BuildRandomRegularishGraph(1 << 13, 8, g, seed=5, symmetrize=True)
    gs.append(g)
    g = CsrGraph()
    BuildRandomGraph(6000, 30000, g, False, seed=9)  # directed: batches never pull
    gs.append(g)
    return gs


def _queries(gs, count, seed):
    rng = np.random.default_rng(seed)
    gid = rng.integers(0, len(gs), count).astype(np.int32)
    src = np.empty(count, np.int32)
    for i, g in enumerate(gs):
        pool = sample_sources(g, 256, seed=seed + i)
        sel = gid == i
        src[sel] = pool[rng.integers(0, pool.size, int(sel.sum()))]
    lim = np.where(rng.random(count) < 0.8, -1, rng.integers(2, 9, count)).astype(np.int32)
    return gid, src, lim


def _oracle(g, s, lim):
    labels, depth = oracle.bfs(g.row_offsets, g.column_indices, int(s), int(lim))
    return labels, depth


@pytest.mark.parametrize("single_strategy", [N.DIRECTION_OPTIMIZING, N.EXPAND_CONTRACT, -1])
def test_mixed_stream_matches_oracle(single_strategy):
    gs = _graphs()
    gid, src, lim = _queries(gs, 240, seed=11)
    with BfsServer(single_strategy=single_strategy) as srv:
        ids = [srv.add_graph(g) for g in gs]
        assert ids == list(range(len(gs)))
        outs, tickets = [], []
        # one common arrival time a little ahead, so the queries meet in the
        # queues and get batched whatever the submission pace
        when = srv.now_ns() + 200_000_000
        for i in range(gid.size):
            out = np.empty(gs[gid[i]].nodes, np.int32)
            outs.append(out)
            tickets.append(srv.submit(int(gid[i]), int(src[i]), int(lim[i]), labels=out, arrival_ns=when))
        srv.drain()
        recs = srv.results(0, gid.size)
        assert (recs["status"] == 0).all()
        assert recs["batch_size"].max() > 1, "no query was batched"
        for i in range(gid.size):
            want, depth = _oracle(gs[gid[i]], src[i], lim[i])
            bad = oracle.compare_labels(outs[i], want)
            assert bad == -1, f"query {i} (graph {gid[i]}, src {src[i]}, limit {lim[i]}): vertex {bad}"
            assert recs["search_depth"][i] == depth, i
        c = srv.counters()
        assert c["completed"] == gid.size and c["failed"] == 0
        assert c["batched_queries"] + c["single_queries"] == gid.size


def test_answers_equal_searches_alone():
    """The same queries through one CsrProblem per graph, one at a time."""
    gs = _graphs()
    gid, src, lim = _queries(gs, 60, seed=23)
    alone = []
    for i in range(gid.size):
        p = CsrProblem.from_graph(gs[gid[i]])
        alone.append(search(p, int(src[i]), strategy=N.DIRECTION_OPTIMIZING, depth_limit=int(lim[i])))
        p.Destroy()
    with BfsServer() as srv:
        for g in gs:
            srv.add_graph(g)
        outs = [np.empty(gs[gid[i]].nodes, np.int32) for i in range(gid.size)]
        for i in range(gid.size):
            srv.submit(int(gid[i]), int(src[i]), int(lim[i]), labels=outs[i])
        srv.drain()
    for i in range(gid.size):
        assert oracle.compare_labels(outs[i], alone[i]) == -1, i


def test_budget_admission_and_accounting():
    import torch
    gs = _graphs()
    b0 = BfsServer.plan_bytes(gs[0].nodes, gs[0].edges, 64)
    b1_8 = BfsServer.plan_bytes(gs[1].nodes, gs[1].edges, 8)
    b1_16 = BfsServer.plan_bytes(gs[1].nodes, gs[1].edges, 16)
    assert b1_8 < b1_16
    budget = b0 + b1_8 + (b1_16 - b1_8) // 2  # graph 1 fits at width 8, not 16
    with BfsServer(memory_budget_bytes=budget) as srv:
        free0 = torch.cuda.mem_get_info()[0]
        g0 = srv.add_graph(gs[0])
        free1 = torch.cuda.mem_get_info()[0]
        bytes0, w0 = srv.graph_info(g0)
        assert (bytes0, w0) == (b0, 64)
        # what the driver reports taken: at most the accounted bytes plus allocation
        # rounding and the kernels' code loaded on first use
        assert free0 - free1 <= bytes0 + (64 << 20)
        g1 = srv.add_graph(gs[1])
        assert srv.graph_info(g1) == (b1_8, 8)
        with pytest.raises(B40cError) as e:
            srv.add_graph(gs[2])
        assert e.value.status == N.ERROR_MEMORY_ALLOCATION
        c = srv.counters()
        assert c["graphs"] == 2 and c["memory_used_bytes"] == b0 + b1_8 and c["memory_budget_bytes"] == budget
        # a width-8 graph still answers 20 queries (in batches of at most 8)
        srcs = sample_sources(gs[1], 20, seed=2)
        t = srv.submit_many(np.full(20, g1, np.int32), srcs)
        srv.drain()
        recs = srv.results(int(t[0]), 20)
        assert (recs["status"] == 0).all() and recs["batch_size"].max() <= 8
        for r, s in zip(recs, srcs):
            assert r["search_depth"] == _oracle(gs[1], s, -1)[1]
        # removing a graph returns its bytes to the budget, and the freed bytes
        # widen the remaining graph's batches again
        srv.remove_graph(g0)
        _, w1 = srv.graph_info(g1)
        assert w1 > 8 and BfsServer.plan_bytes(gs[1].nodes, gs[1].edges, w1) <= budget
        assert srv.counters()["memory_used_bytes"] == BfsServer.plan_bytes(gs[1].nodes, gs[1].edges, w1)
        t = srv.submit_many(np.full(w1, g1, np.int32), sample_sources(gs[1], w1, seed=3))
        srv.drain()
        recs = srv.results(int(t[0]), w1)
        assert (recs["status"] == 0).all() and recs["batch_size"].max() > 8
        srv.remove_graph(g1)
        assert srv.counters()["memory_used_bytes"] == 0
        assert srv.add_graph(gs[2]) == 2


def test_remove_refused_while_pending():
    gs = _graphs()
    with BfsServer() as srv:
        g = srv.add_graph(gs[0])
        t = srv.submit(g, int(sample_sources(gs[0], 1)[0]), arrival_ns=srv.now_ns() + 300_000_000)
        with pytest.raises(B40cError) as e:
            srv.remove_graph(g)
        assert e.value.status == N.ERROR_NOT_READY
        assert srv.result(t)["status"] == N.ERROR_NOT_READY
        r = srv.wait(t)
        assert r["status"] == 0 and r["launch_ns"] >= r["arrival_ns"]
        srv.remove_graph(g)


def test_timed_arrivals_wait_for_their_time():
    gs = _graphs()
    gid, src, lim = _queries(gs, 400, seed=31)
    with BfsServer() as srv:
        for g in gs:
            srv.add_graph(g)
        t0 = srv.now_ns() + 5_000_000
        arrivals = t0 + np.sort(np.random.default_rng(1).integers(0, 60_000_000, gid.size))
        tickets = srv.submit_many(gid, src, lim, arrivals)
        srv.drain()
        recs = srv.results(int(tickets[0]), gid.size)
    assert (recs["status"] == 0).all()
    assert (recs["launch_ns"] >= recs["arrival_ns"]).all()
    assert (recs["finish_ns"] > recs["launch_ns"]).all()
    s = latency_summary(recs)
    assert s["queries"] == gid.size and s["p99_ms"] >= s["p50_ms"] > 0
    for i in range(0, gid.size, 7):
        assert recs["search_depth"][i] == _oracle(gs[gid[i]], src[i], lim[i])[1]


def test_bad_queries_rejected():
    gs = _graphs()
    with BfsServer() as srv:
        g = srv.add_graph(gs[0])
        with pytest.raises(B40cError):
            srv.submit(g + 1, 0)
        with pytest.raises(B40cError):
            srv.submit(g, gs[0].nodes)
        with pytest.raises(B40cError):
            srv.submit_many([g, g], [0, -1])
        assert srv.counters()["submitted"] == 0


def test_batches_of_different_graphs_overlap_on_the_device():
    """Each in-flight slot has its own stream and a share of every SM: batches
    of two graphs issued together run at the same time on the GPU (their
    device-clock intervals intersect), and their answers stay exact."""
    gs = _graphs()[:3]
    with BfsServer(max_in_flight=2) as srv:
        for g in gs:
            srv.add_graph(g)
        rng = np.random.default_rng(4)
        gid = np.repeat(np.arange(3, dtype=np.int32), 192)
        src = np.concatenate([sample_sources(g, 192, seed=i) for i, g in enumerate(gs)])
        order = rng.permutation(gid.size)
        gid, src = gid[order], src[order]
        t = srv.submit_many(gid, src, None, np.full(gid.size, srv.now_ns() + 50_000_000, np.int64))
        srv.drain()
        recs = srv.results(int(t[0]), gid.size)
    assert (recs["status"] == 0).all()
    assert (recs["gpu_end_ns"] > recs["gpu_start_ns"]).all()
    spans = {(int(r["graph"]), int(r["gpu_start_ns"]), int(r["gpu_end_ns"])) for r in recs}
    spans = sorted(spans, key=lambda x: x[1])
    overlaps = sum(1 for i, a in enumerate(spans) for b in spans[i + 1:]
                   if b[1] < a[2] and a[0] != b[0])
    assert overlaps > 0, "no two batches of different graphs ran at the same time"
    for i in range(0, gid.size, 17):
        want, depth = _oracle(gs[gid[i]], src[i], -1)
        assert recs["search_depth"][i] == depth


def test_queries_join_a_running_batch_with_exact_labels():
    """Queries that arrive while their graph's batched search runs join it at
    a level boundary (free slots of the batch) instead of waiting for the next
    batch; each still gets exactly the labels of its search alone."""
    g = CsrGraph()
    BuildGrid2dGraph(1000, g)  # about 2,000 levels: the batch runs for many milliseconds
    y, x = np.divmod(np.arange(g.nodes), 1000)
    with BfsServer(max_batch=8, max_in_flight=1) as srv:
        gid = srv.add_graph(g)
        t0 = srv.now_ns() + 20_000_000
        first = [0, 999]
        later = [500_500, 999_999, 1234, 777_000]
        import torch
        # pageable arrays for the first queries (copied when their batch retires),
        # page-locked ones for the joining queries (copies queued behind the search)
        outs = {s: np.empty(g.nodes, np.int32) for s in first}
        outs.update({s: torch.empty(g.nodes, dtype=torch.int32, pin_memory=True).numpy() for s in later})
        tickets = {}
        for s in first:
            tickets[s] = srv.submit(gid, s, -1, labels=outs[s], arrival_ns=t0)
        # the late queries arrive once the first batch is on the device (a batch
        # of this graph runs for many milliseconds)
        import time
        deadline = time.monotonic() + 30
        while srv.counters()["batches"] < 1 and time.monotonic() < deadline:
            time.sleep(0.0002)
        assert srv.counters()["batches"] == 1
        for k, s in enumerate(later):
            tickets[s] = srv.submit(gid, s, 3 if k == 2 else -1, labels=outs[s], arrival_ns=srv.now_ns())
        srv.drain()
        recs = {s: srv.result(t) for s, t in tickets.items()}
        c = srv.counters()
    assert all(r["status"] == 0 for r in recs.values())
    assert c["joined_queries"] >= 1, c
    joined = [s for s in later if recs[s]["launch_ns"] > recs[first[0]]["launch_ns"] and
              recs[s]["batch_size"] == recs[first[0]]["batch_size"]]
    assert joined, "no late query shared the first batch"
    for k, s in enumerate(first + later):
        sy, sx = divmod(s, 1000)
        want = (np.abs(x - sx) + np.abs(y - sy)).astype(np.int32)
        if s == later[2]:
            want = np.where(want <= 3, want, -1).astype(np.int32)
        assert np.array_equal(outs[s], want), f"source {s}"
        assert recs[s]["search_depth"] == int(want.max()) + 1
