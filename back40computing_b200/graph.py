"""Host graph container and builders (b40c/graph/csr_graph.cuh, builder/*.cuh).

``CsrGraph`` mirrors the reference's ``CsrGraph<VertexId, Value, SizeT>``
(csr_graph.cuh:51-245) with int32 vertex ids and offsets; the builders call
the library's native multi-threaded builders through the C ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

from . import _native as N


class CsrGraph:
    """Host CSR graph: ``row_offsets[nodes + 1]``, ``column_indices[edges]``."""

    def __init__(self, pinned: bool = False):
        self.nodes = 0
        self.edges = 0
        self.row_offsets: np.ndarray | None = None
        self.column_indices: np.ndarray | None = None
        self.values = None
        self.pinned = pinned
        self._csr: N.Csr | None = None  # native storage backing the arrays

    # csr_graph.cuh:76-102
    def FromScratch(self, nodes: int, edges: int) -> None:
        self.Free()
        self.nodes, self.edges = int(nodes), int(edges)
        self.row_offsets = np.zeros(self.nodes + 1, dtype=np.int32)
        self.column_indices = np.zeros(self.edges, dtype=np.int32)

    # csr_graph.cuh:109-152 (stable by-row ordering)
    def FromCoo(self, rows, cols, nodes: int, ordered_rows: bool = False) -> None:
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        csr = N.Csr()
        N.check(N.lib().b40c_csr_from_coo(N.i32p(rows), N.i32p(cols), int(nodes), int(rows.size),
                                          int(self.pinned), C.byref(csr)), "b40c_csr_from_coo")
        self._adopt(csr)

    def _adopt(self, csr: N.Csr) -> None:
        self.Free()
        self._csr = csr
        self.nodes, self.edges = int(csr.nodes), int(csr.edges)
        self.row_offsets = np.ctypeslib.as_array(csr.row_offsets, shape=(self.nodes + 1,))
        self.column_indices = np.ctypeslib.as_array(csr.column_indices, shape=(max(self.edges, 1),))[: self.edges]

    @classmethod
    def from_arrays(cls, row_offsets, column_indices) -> "CsrGraph":
        g = cls()
        g.row_offsets = np.ascontiguousarray(row_offsets, dtype=np.int32)
        g.column_indices = np.ascontiguousarray(column_indices, dtype=np.int32)
        g.nodes = g.row_offsets.size - 1
        g.edges = g.column_indices.size
        return g

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_offsets).astype(np.int64)

    # csr_graph.cuh:157-190
    def PrintHistogram(self) -> str:
        deg = self.degrees()
        logs = np.full(deg.shape, -1, dtype=np.int64)
        nz = deg > 0
        logs[nz] = np.floor(np.log2(deg[nz])).astype(np.int64)
        top = int(logs.max()) if logs.size else -1
        lines = [f"Degree Histogram ({self.nodes} vertices, {self.edges} directed edges):"]
        for i in range(-1, top + 1):
            c = int((logs == i).sum())
            lines.append(f"\tDegree 2^{i}: {c} ({100.0 * c / max(self.nodes, 1):.2f}%)")
        text = "\n".join(lines)
        print(text)
        return text

    # csr_graph.cuh:196-210
    def DisplayGraph(self) -> None:
        print("Input Graph:")
        for v in range(self.nodes):
            nb = self.column_indices[self.row_offsets[v]:self.row_offsets[v + 1]]
            print(f"{v}: " + "".join(f"{int(x)}, " for x in nb))

    # csr_graph.cuh:214-236
    def Free(self) -> None:
        if self._csr is not None:
            N.lib().b40c_graph_free(C.byref(self._csr))
            self._csr = None
        self.row_offsets = None
        self.column_indices = None
        self.nodes = self.edges = 0

    def __del__(self):
        try:
            self.Free()
        except Exception:
            pass


# ---- builders (b40c/graph/builder/*.cuh); return 0 on success like the reference ----

def _build(fn_name: str, graph: CsrGraph, *args) -> int:
    csr = N.Csr()
    N.check(getattr(N.lib(), fn_name)(*args, int(graph.pinned), C.byref(csr)), fn_name)
    graph._adopt(csr)
    return 0


def BuildGrid2dGraph(width: int, graph: CsrGraph) -> int:
    """grid2d.cuh:54-114: width x width lattice with a self-loop per vertex."""
    return _build("b40c_build_grid2d", graph, int(width))


def BuildGrid3dGraph(width: int, graph: CsrGraph) -> int:
    """grid3d.cuh:54-129: width^3 lattice with a self-loop per vertex."""
    return _build("b40c_build_grid3d", graph, int(width))


def BuildRmatGraph(nodes: int, edges: int, graph: CsrGraph, undirected: bool, a: float, b: float, c: float,
                   seed: int = 0, permute: bool = False) -> int:
    """rmat.cuh:128-206 with a seeded generator (and an optional vertex permutation)."""
    return _build("b40c_build_rmat", graph, int(nodes), int(edges), int(bool(undirected)), float(a), float(b),
                  float(c), int(seed), int(bool(permute)))


def BuildRandomGraph(nodes: int, edges: int, graph: CsrGraph, undirected: bool, seed: int = 0) -> int:
    """random.cuh:54-98 with a seeded generator."""
    return _build("b40c_build_random", graph, int(nodes), int(edges), int(bool(undirected)), int(seed))


def BuildRandomRegularishGraph(nodes: int, degree: int, graph: CsrGraph, seed: int = 0,
                               symmetrize: bool = False) -> int:
    """rr.cuh:53-91 with a seeded generator; optionally symmetrised."""
    return _build("b40c_build_rr", graph, int(nodes), int(degree), int(bool(symmetrize)), int(seed))


def _read(fn_name: str, graph: CsrGraph, path, *args) -> int:
    """Runs a reader; returns 0, or -1 with the parse error printed (the
    reference builders' convention)."""
    csr = N.Csr()
    p = None if path is None else os.fsencode(path)
    rc = getattr(N.lib(), fn_name)(p, *args, int(graph.pinned), C.byref(csr))
    if rc != N.SUCCESS:
        print(f"{fn_name}: {N.lib().b40c_last_error_string().decode(errors='replace')}", file=sys.stderr)
        return -1
    graph._adopt(csr)
    return 0


def BuildMarketGraph(path, graph: CsrGraph, undirected: bool) -> int:
    """market.cuh:180-208 (ReadMarketStream :49-160).  path None = stdin."""
    return _read("b40c_read_market", graph, path, int(bool(undirected)))


def BuildDimacsGraph(path, graph: CsrGraph, undirected: bool, splice: int = 0) -> int:
    """dimacs.cuh:235-283 (ReadDimacsStream :52-228); splice > 0 reads path.0, path.1, ..."""
    return _read("b40c_read_dimacs", graph, path, int(bool(undirected)), int(splice))


def BuildMetisGraph(path, graph: CsrGraph) -> int:
    """metis.cuh:193-230 (ReadMetisStream :51-187).  path None = stdin."""
    return _read("b40c_read_metis", graph, path)


def sample_sources(graph: CsrGraph, count: int, seed: int = 0) -> np.ndarray:
    """`count` distinct seeded sources among vertices with nonzero degree."""
    csr = N.Csr()
    csr.nodes, csr.edges = graph.nodes, graph.edges
    csr.row_offsets = N.i32p(graph.row_offsets)
    csr.column_indices = N.i32p(graph.column_indices) if graph.edges else None
    out = np.zeros(int(count), dtype=np.int32)
    N.check(N.lib().b40c_sample_sources(C.byref(csr), int(count), int(seed), N.i32p(out)), "b40c_sample_sources")
    return out
