"""BFS problem and enactors (b40c/graph/bfs), the host-side mirror of the
reference's C++ interface over the C ABI.

* ``CsrProblem``  -- bfs::CsrProblem (csr_problem.cuh:72-756)
* ``EnactorExpandContract`` / ``EnactorContractExpand`` / ``EnactorTwoPhase``
  / ``EnactorHybrid`` -- the four single-GPU enactors, with
  ``EnactFusedSearch`` / ``EnactIterativeSearch`` / ``EnactSearch`` and
  ``GetStatistics`` returning ``(total_queued, search_depth, avg_duty)``.

Methods return the cudaError_t status like the reference (0 on success); the
``*_or_raise`` helpers and ``search()`` raise ``B40cError`` instead.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .graph import CsrGraph

VERTEX_FRONTIERS = N.VERTEX_FRONTIERS
EDGE_FRONTIERS = N.EDGE_FRONTIERS
MIXED_FRONTIERS = N.MIXED_FRONTIERS
MULTI_GPU_FRONTIERS = N.MULTI_GPU_FRONTIERS

EXPAND_CONTRACT = N.EXPAND_CONTRACT
CONTRACT_EXPAND = N.CONTRACT_EXPAND
TWO_PHASE = N.TWO_PHASE
HYBRID = N.HYBRID
DIRECTION_OPTIMIZING = N.DIRECTION_OPTIMIZING

Policy = N.Policy


def default_policy(strategy: int) -> N.Policy:
    pol = N.Policy()
    N.check(N.lib().b40c_bfs_default_policy(int(strategy), C.byref(pol)), "b40c_bfs_default_policy")
    return pol


class CsrProblem:
    """Device-resident CSR plus per-search state (labels, visited mask, queues)."""

    def __init__(self, mark_predecessors: bool = False, device: int = 0):
        self.MARK_PREDECESSORS = bool(mark_predecessors)
        self.device = int(device)
        self.nodes = 0
        self.edges = 0
        self.num_gpus = 0
        self._h = C.c_void_p(None)
        self._keep = None  # host arrays kept alive for stream-from-host
        self._ms_k = 0     # sources of the last batch

    # csr_problem.cuh:328-540
    def FromHostProblem(self, stream_from_host: bool, nodes: int, edges: int, column_indices, row_offsets,
                        num_gpus: int = 1) -> int:
        if num_gpus != 1:
            N.lib()  # loads (and fails loudly) even on the error path
            return N.ERROR_INVALID_VALUE
        self.Destroy()
        ro = np.ascontiguousarray(row_offsets, dtype=np.int32)
        ci = np.ascontiguousarray(column_indices, dtype=np.int32)
        h = C.c_void_p()
        status = N.lib().b40c_bfs_problem_create(N.i32p(ro), N.i32p(ci) if ci.size else None, int(nodes), int(edges),
                                                 int(self.MARK_PREDECESSORS), int(bool(stream_from_host)),
                                                 self.device, C.byref(h))
        if status == N.SUCCESS:
            self._h = h
            self.nodes, self.edges, self.num_gpus = int(nodes), int(edges), 1
            self._keep = (ro, ci) if stream_from_host else None
        return status

    @classmethod
    def from_graph(cls, graph: CsrGraph, mark_predecessors: bool = False, device: int = 0,
                   stream_from_host: bool = False) -> "CsrProblem":
        p = cls(mark_predecessors, device)
        N.check(p.FromHostProblem(stream_from_host, graph.nodes, graph.edges, graph.column_indices,
                                  graph.row_offsets, 1), "FromHostProblem")
        return p

    @classmethod
    def from_coo(cls, rows, cols, nodes: int, mark_predecessors: bool = False, device: int = 0) -> "CsrProblem":
        """A problem from a host COO edge list, converted to CSR on the GPU
        (rows keep their input order, as CsrGraph::FromCoo)."""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        p = cls(mark_predecessors, device)
        h = C.c_void_p()
        N.check(N.lib().b40c_bfs_problem_create_coo(N.i32p(r), N.i32p(c), int(nodes), int(r.size),
                                                    int(bool(mark_predecessors)), int(device), C.byref(h)),
                "b40c_bfs_problem_create_coo")
        p._h = h
        p.nodes, p.edges, p.num_gpus = int(nodes), int(r.size), 1
        return p

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise N.B40cError(N.ERROR_INVALID_VALUE, "problem not initialised (FromHostProblem)")
        return self._h

    # csr_problem.cuh:547-750
    def Reset(self, frontier_type: int, queue_sizing: float = 1.3) -> int:
        return N.lib().b40c_bfs_problem_reset(self.handle, int(frontier_type), float(queue_sizing))

    # csr_problem.cuh:255-322
    def ExtractResults(self, h_labels: np.ndarray) -> int:
        assert h_labels.dtype == np.int32 and h_labels.size >= self.nodes
        return N.lib().b40c_bfs_extract(self.handle, N.i32p(h_labels))

    def ExtractResultsAsync(self, h_labels: np.ndarray, slot: int) -> int:
        """Starts the read-back of the last search's labels into h_labels through
        staging slot 0 or 1 and returns at once (pinned memory overlaps the copy
        with the next search); ExtractWait(slot) completes it.  h_labels must
        stay alive and untouched until then."""
        assert h_labels.dtype == np.int32 and h_labels.size >= self.nodes
        return N.lib().b40c_bfs_extract_async(self.handle, N.i32p(h_labels), int(slot))

    def ExtractWait(self, slot: int) -> int:
        return N.lib().b40c_bfs_extract_wait(self.handle, int(slot))

    def labels(self) -> np.ndarray:
        out = np.empty(self.nodes, dtype=np.int32)
        N.check(self.ExtractResults(out), "ExtractResults")
        return out

    def set_stream(self, stream_handle: int | None) -> None:
        N.check(N.lib().b40c_bfs_set_stream(self.handle, C.c_void_p(stream_handle or None)), "set_stream")

    def last_elapsed_ms(self) -> float:
        ms = C.c_float(0)
        N.check(N.lib().b40c_bfs_last_elapsed_ms(self.handle, C.byref(ms)), "last_elapsed_ms")
        return float(ms.value)

    def recent_search_ms(self, count: int) -> np.ndarray:
        out = (C.c_float * int(count))()
        N.check(N.lib().b40c_bfs_recent_search_ms(self.handle, int(count), out), "recent_search_ms")
        return np.array(out[:], dtype=np.float64)

    def set_instrument(self, on: bool = True) -> None:
        N.check(N.lib().b40c_bfs_set_instrument(self.handle, int(bool(on))), "set_instrument")

    def level_records(self, max_records: int = 1 << 16) -> list[dict]:
        """Per-pass records of the last instrumented search (with durations)."""
        buf = (N.LevelRecord * (max_records + 1))()
        cnt = C.c_int32(0)
        N.check(N.lib().b40c_bfs_level_records(self.handle, buf, max_records + 1, C.byref(cnt)), "level_records")
        recs = [dict(vertices=r.vertices, edges=r.edges, bottom_up=bool(r.bottom_up), pass_=r.pass_,
                     t_ns=int(r.t_ns)) for r in buf[:cnt.value]]
        for a, b in zip(recs, recs[1:]):
            a["ns"] = b["t_ns"] - a["t_ns"]
        return [r for r in recs if r["pass_"] >= 0]

    def cta_arrivals(self, max_passes: int = 64, phases: bool = False) -> np.ndarray:
        """[pass, cta] end-of-level barrier arrival times (ns) of the last
        instrumented persistent search (0 where a CTA did not arrive); with
        phases=True [pass, cta, 8] including the in-level phase stamps."""
        buf = np.zeros(max_passes * 2048 * 8, dtype=np.uint64)
        g = C.c_int32(0)
        N.check(N.lib().b40c_bfs_cta_arrivals(self.handle, buf.ctypes.data_as(C.POINTER(C.c_uint64)),
                                              int(max_passes), C.byref(g)), "cta_arrivals")
        a = buf[:max_passes * g.value * 8].reshape(max_passes, g.value, 8)
        return a if phases else a[:, :, 7]

    # ---- batched multi-source searches ------------------------------------------------
    def msbfs(self, sources, depth_limits=None, policy: N.Policy | None = None, max_grid_size: int = 0) -> None:
        """Searches up to 64 sources together (asynchronous); see labels_of()."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        lim = None if depth_limits is None else np.ascontiguousarray(depth_limits, dtype=np.int32)
        pol = C.byref(policy) if policy is not None else None
        N.check(N.lib().b40c_msbfs_enact(self.handle, N.i32p(src), N.i32p(lim) if lim is not None else None,
                                         int(src.size), int(max_grid_size), pol), "msbfs")
        self._ms_k = int(src.size)

    def msbfs_join(self, slot: int, source: int, depth_limit: int = -1) -> None:
        """Adds `source` in slot `slot` to the batch in flight (taken at its next
        level boundary; see msbfs_joined)."""
        N.check(N.lib().b40c_msbfs_join(self.handle, int(slot), int(source), int(depth_limit)), "b40c_msbfs_join")

    def msbfs_joined(self) -> tuple[int, np.ndarray]:
        """(join requests the last batch took, every slot's search depth [64])."""
        taken = C.c_int32(0)
        depths = np.zeros(64, np.int32)
        N.check(N.lib().b40c_msbfs_joined(self.handle, C.byref(taken), N.i32p(depths)), "b40c_msbfs_joined")
        return taken.value, depths

    def labels_of(self, slot: int) -> np.ndarray:
        """Labels of source `slot` of the last batch."""
        out = np.empty(self.nodes, dtype=np.int32)
        N.check(N.lib().b40c_msbfs_extract(self.handle, int(slot), N.i32p(out)), "msbfs_extract")
        return out

    def msbfs_depths(self) -> np.ndarray:
        """Search depth (max label + 1) of every slot of the last batch."""
        out = np.empty(64, dtype=np.int32)
        N.check(N.lib().b40c_msbfs_stats(self.handle, N.i32p(out)), "msbfs_stats")
        return out[:self._ms_k]

    def is_symmetric(self) -> bool:
        out = C.c_int32(0)
        N.check(N.lib().b40c_bfs_problem_is_symmetric(self.handle, C.byref(out)), "is_symmetric")
        return bool(out.value)

    def device_view(self) -> N.DeviceView:
        v = N.DeviceView()
        N.check(N.lib().b40c_bfs_device_view_get(self.handle, C.byref(v)), "device_view")
        return v

    def Destroy(self) -> None:
        if self._h:
            N.lib().b40c_bfs_problem_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass


class _Enactor:
    STRATEGY = -1
    FRONTIER = VERTEX_FRONTIERS

    def __init__(self, DEBUG: bool = False, policy: N.Policy | None = None):
        self.DEBUG = DEBUG
        self.policy = policy
        self._problem: CsrProblem | None = None

    def GetFrontierType(self) -> int:
        return self.FRONTIER

    def _enact(self, problem: CsrProblem, src: int, mode: int, max_grid_size: int, depth_limit: int = -1) -> int:
        self._problem = problem
        pol = C.byref(self.policy) if self.policy is not None else None
        return N.lib().b40c_bfs_enact_limited(problem.handle, self.STRATEGY, int(mode), int(src), int(depth_limit),
                                              int(max_grid_size), pol)

    def EnactFusedSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return self._enact(problem, src, N.ENACT_FUSED, max_grid_size)

    def EnactIterativeSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return self._enact(problem, src, N.ENACT_ITERATIVE, max_grid_size)

    def EnactGraphSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return self._enact(problem, src, N.ENACT_GRAPH, max_grid_size)

    def GetStatistics(self) -> tuple[int, int, float]:
        if self._problem is None:
            return 0, 0, 0.0
        tq, depth, duty = C.c_int64(0), C.c_int32(0), C.c_double(0)
        N.check(N.lib().b40c_bfs_stats(self._problem.handle, C.byref(tq), C.byref(depth), C.byref(duty)),
                "GetStatistics")
        return int(tq.value), int(depth.value), float(duty.value)


class EnactorExpandContract(_Enactor):
    """enactor_expand_contract.cuh:59 -- vertex frontiers, fused expand+contract."""
    STRATEGY = EXPAND_CONTRACT
    FRONTIER = VERTEX_FRONTIERS


class EnactorContractExpand(_Enactor):
    """enactor_contract_expand.cuh:61 -- edge frontiers, fused contract+expand."""
    STRATEGY = CONTRACT_EXPAND
    FRONTIER = EDGE_FRONTIERS


class EnactorTwoPhase(_Enactor):
    """enactor_two_phase.cuh:68 -- separate contract and expand kernels per level."""
    STRATEGY = TWO_PHASE
    FRONTIER = MIXED_FRONTIERS


class EnactorHybrid(_Enactor):
    """enactor_hybrid.cuh:64 -- fused contract-expand, two-phase while saturated."""
    STRATEGY = HYBRID
    FRONTIER = EDGE_FRONTIERS

    def EnactSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return self._enact(problem, src, N.ENACT_FUSED, max_grid_size)


class EnactorDirectionOptimizing(_Enactor):
    """No counterpart in the reference: top-down expand-contract levels plus
    bottom-up levels while the frontier is large (undirected graphs only; a
    directed graph runs plain expand-contract).  Same labels as the others."""
    STRATEGY = DIRECTION_OPTIMIZING
    FRONTIER = VERTEX_FRONTIERS


ENACTORS = {
    EXPAND_CONTRACT: EnactorExpandContract,
    CONTRACT_EXPAND: EnactorContractExpand,
    TWO_PHASE: EnactorTwoPhase,
    HYBRID: EnactorHybrid,
    DIRECTION_OPTIMIZING: EnactorDirectionOptimizing,
}


def search(problem: CsrProblem, src: int, strategy: int = EXPAND_CONTRACT, mode: int = N.ENACT_FUSED,
           depth_limit: int = -1, queue_sizing: float = 1.3, policy: N.Policy | None = None,
           max_grid_size: int = 0) -> np.ndarray:
    """Reset + one search + extract; raises on any failure.  Returns labels[n]."""
    enactor = ENACTORS[strategy](policy=policy)
    N.check(problem.Reset(enactor.GetFrontierType(), queue_sizing), "Reset")
    N.check(enactor._enact(problem, src, mode, max_grid_size, depth_limit), "Enact")
    return problem.labels()
