"""BFS query server over several resident graphs (include/b40c_server.h).

The reference answers one query at a time from its test driver
(test/bfs/test_bfs.cu:584-783); this server keeps graphs resident inside a
device-memory budget and answers single-source (optionally depth-limited)
queries with continuous batching on the native dispatcher thread.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .graph import CsrGraph


class BfsServer:
    """Python face of ``b40c_server``.

    ``submit`` returns a ticket; ``wait``/``result`` give the query's record
    (status, search depth, batch size, arrival / launch / finish times on the
    server clock); labels are delivered into the caller's array when one is
    passed.  ``submit_many`` queues a whole timed request stream in one call.
    """

    def __init__(self, device: int = 0, memory_budget_bytes: int = 0, max_batch: int = 0,
                 single_strategy: int = N.DIRECTION_OPTIMIZING, max_in_flight: int = 0, ctas_per_sm: int = 0):
        o = N.ServerOptions()
        o.memory_budget_bytes = int(memory_budget_bytes)
        o.max_batch = int(max_batch)
        o.single_strategy = int(single_strategy)
        o.max_in_flight = int(max_in_flight)
        o.ctas_per_sm = int(ctas_per_sm)
        self._h = C.c_void_p(None)
        N.check(N.lib().b40c_server_create(int(device), C.byref(o), C.byref(self._h)), "b40c_server_create")
        self._labels = {}  # ticket -> caller array kept alive until the query finishes

    @property
    def handle(self):
        if not self._h:
            raise N.B40cError(N.ERROR_INVALID_VALUE, "server closed")
        return self._h

    def add_graph(self, graph: CsrGraph) -> int:
        gid = C.c_int32(-1)
        N.check(N.lib().b40c_server_add_graph(self.handle, N.i32p(graph.row_offsets), N.i32p(graph.column_indices),
                                              int(graph.nodes), int(graph.edges), C.byref(gid)),
                "b40c_server_add_graph")
        return gid.value

    def set_graph_policy(self, graph_id: int, single: N.Policy | None = None, batch: N.Policy | None = None) -> None:
        N.check(N.lib().b40c_server_set_graph_policy(self.handle, int(graph_id),
                                                     C.byref(single) if single is not None else None,
                                                     C.byref(batch) if batch is not None else None),
                "b40c_server_set_graph_policy")

    def add_tuned_graph(self, graph: CsrGraph) -> int:
        """add_graph plus the autotuner's policies for the graph's class."""
        from . import autotune
        gid = self.add_graph(graph)
        cls = autotune.classify(graph)
        self.set_graph_policy(gid, autotune.policy_for(cls, "direction-optimizing"), autotune.policy_for(cls, "batched"))
        return gid

    def remove_graph(self, graph_id: int) -> None:
        N.check(N.lib().b40c_server_remove_graph(self.handle, int(graph_id)), "b40c_server_remove_graph")

    def graph_info(self, graph_id: int) -> tuple[int, int]:
        """(device bytes held, batch width)."""
        b, w = C.c_int64(0), C.c_int32(0)
        N.check(N.lib().b40c_server_graph_info(self.handle, int(graph_id), C.byref(b), C.byref(w)), "graph_info")
        return b.value, w.value

    @staticmethod
    def plan_bytes(nodes: int, edges: int, max_batch: int) -> int:
        b = C.c_int64(0)
        N.check(N.lib().b40c_server_plan_bytes(int(nodes), int(edges), int(max_batch), C.byref(b)), "plan_bytes")
        return b.value

    def now_ns(self) -> int:
        t = C.c_int64(0)
        N.check(N.lib().b40c_server_now_ns(self.handle, C.byref(t)), "now_ns")
        return t.value

    def submit(self, graph_id: int, source: int, depth_limit: int = -1, labels: np.ndarray | None = None,
               arrival_ns: int = -1) -> int:
        ptr = None
        if labels is not None:
            assert labels.dtype == np.int32 and labels.flags["C_CONTIGUOUS"]
            ptr = C.c_void_p(labels.ctypes.data)
        t = C.c_int64(-1)
        N.check(N.lib().b40c_server_submit(self.handle, int(graph_id), int(source), int(depth_limit), ptr,
                                           int(arrival_ns), C.byref(t)), "b40c_server_submit")
        if labels is not None:
            self._labels[t.value] = labels
        return t.value

    def submit_many(self, graph_ids, sources, depth_limits=None, arrival_ns=None) -> np.ndarray:
        g = np.ascontiguousarray(graph_ids, dtype=np.int32)
        s = np.ascontiguousarray(sources, dtype=np.int32)
        lim = None if depth_limits is None else np.ascontiguousarray(depth_limits, dtype=np.int32)
        arr = None if arrival_ns is None else np.ascontiguousarray(arrival_ns, dtype=np.int64)
        tickets = np.empty(g.size, dtype=np.int64)
        N.check(N.lib().b40c_server_submit_many(
            self.handle, int(g.size), N.i32p(g), N.i32p(s), N.i32p(lim) if lim is not None else None,
            arr.ctypes.data_as(C.POINTER(C.c_int64)) if arr is not None else None,
            tickets.ctypes.data_as(C.POINTER(C.c_int64))), "b40c_server_submit_many")
        return tickets

    @staticmethod
    def _record(r: N.ServerResult) -> dict:
        return {name: getattr(r, name) for name, _ in N.ServerResult._fields_}

    def result(self, ticket: int) -> dict:
        r = N.ServerResult()
        N.check(N.lib().b40c_server_result_get(self.handle, int(ticket), C.byref(r)), "result_get")
        return self._record(r)

    def wait(self, ticket: int) -> dict:
        r = N.ServerResult()
        N.check(N.lib().b40c_server_wait(self.handle, int(ticket), C.byref(r)), "b40c_server_wait")
        self._labels.pop(int(ticket), None)
        return self._record(r)

    def drain(self) -> None:
        N.check(N.lib().b40c_server_drain(self.handle), "b40c_server_drain")
        self._labels.clear()

    def results(self, first: int, count: int) -> np.ndarray:
        out = np.zeros(int(count), dtype=N.SERVER_RESULT_DTYPE)
        N.check(N.lib().b40c_server_results(self.handle, int(first), int(count), C.c_void_p(out.ctypes.data)),
                "b40c_server_results")
        return out

    def counters(self) -> dict:
        c = N.ServerCounters()
        N.check(N.lib().b40c_server_counters_get(self.handle, C.byref(c)), "counters")
        return {name: getattr(c, name) for name, _ in N.ServerCounters._fields_ if name != "reserved"}

    def close(self) -> None:
        if self._h:
            N.lib().b40c_server_destroy(self._h)
            self._h = C.c_void_p(None)
            self._labels.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def latency_summary(records: np.ndarray) -> dict:
    """p50 / p99 / mean end-to-end latency (finish - arrival) in ms and the
    throughput over the span from the first arrival to the last finish."""
    ok = records[records["status"] == 0]
    lat = (ok["finish_ns"] - ok["arrival_ns"]) / 1e6
    span_s = (records["finish_ns"].max() - records["arrival_ns"].min()) / 1e9 if records.size else 0.0
    return {
        "queries": int(records.size), "failed": int((records["status"] != 0).sum()),
        "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
        "mean_ms": float(lat.mean()) if lat.size else None,
        "queries_per_s": float(records.size / span_s) if span_s > 0 else None,
        "mean_batch": float(ok["batch_size"].mean()) if ok.size else None,
    }
