"""CPU oracle bindings.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only as the checker or the timed CPU baseline; the product
library never calls it.

* ``liboracle.so``  -- the C restatement of the reference's serial CPU BFS
  and validators (bfs_oracle.c, citing test/bfs/test_bfs.cu line ranges).
* ``_ref/libb40c_ref.so`` -- the reference's own host code (its builders and
  SimpleReferenceBfs) compiled from the reference tree by build_ref.sh, when
  that tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libb40c_ref.so")

_P32 = C.POINTER(C.c_int32)
_P64 = C.POINTER(C.c_int64)
_o = None
_r = None


def _p32(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P32)


def olib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run python -m back40computing_b200.build")
        L = C.CDLL(ORACLE_LIB)
        L.oracle_bfs.restype = C.c_int64
        L.oracle_bfs.argtypes = [C.c_int64, _P32, _P32, C.c_int32, _P32]
        L.oracle_bfs_limited.restype = C.c_int64
        L.oracle_bfs_limited.argtypes = [C.c_int64, _P32, _P32, C.c_int32, C.c_int32, _P32]
        L.oracle_check_predecessors.restype = C.c_int64
        L.oracle_check_predecessors.argtypes = [C.c_int64, _P32, _P32, _P32, _P32, _P32]
        L.oracle_visited_stats.restype = None
        L.oracle_visited_stats.argtypes = [C.c_int64, _P32, _P32, _P64, _P64]
        L.oracle_compare_labels.restype = C.c_int64
        L.oracle_compare_labels.argtypes = [C.c_int64, _P32, _P32]
        L.oracle_level_histogram.restype = C.c_int64
        L.oracle_level_histogram.argtypes = [C.c_int64, _P32, _P64, C.c_int64]
        _o = L
    return _o


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def rlib():
    global _r
    if _r is None:
        if not have_ref():
            raise ImportError(f"{REF_LIB} missing (built from the reference tree by oracle/build_ref.sh)")
        L = C.CDLL(REF_LIB)
        PP = C.POINTER(_P32)
        L.ref_simple_bfs.restype = C.c_int
        L.ref_simple_bfs.argtypes = [C.c_int32, C.c_int32, _P32, _P32, C.c_int32, _P32, _P64,
                                     C.POINTER(C.c_double)]
        for name in ("ref_build_grid2d", "ref_build_grid3d"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [C.c_int32, PP, PP, _P64, _P64]
        L.ref_build_rmat.restype = C.c_int
        L.ref_build_rmat.argtypes = [C.c_int32, C.c_int32, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint,
                                     PP, PP, _P64, _P64]
        L.ref_build_random.restype = C.c_int
        L.ref_build_random.argtypes = [C.c_int32, C.c_int32, C.c_int, C.c_uint, PP, PP, _P64, _P64]
        L.ref_build_rr.restype = C.c_int
        L.ref_build_rr.argtypes = [C.c_int32, C.c_int32, C.c_uint, PP, PP, _P64, _P64]
        L.ref_random_node.restype = C.c_int32
        L.ref_random_node.argtypes = [C.c_int32, C.c_uint, C.c_int]
        L.ref_read_market.restype = C.c_int
        L.ref_read_market.argtypes = [C.c_char_p, C.c_int, PP, PP, _P64, _P64]
        L.ref_read_dimacs.restype = C.c_int
        L.ref_read_dimacs.argtypes = [C.c_char_p, C.c_int, C.c_int, PP, PP, _P64, _P64]
        L.ref_read_metis.restype = C.c_int
        L.ref_read_metis.argtypes = [C.c_char_p, PP, PP, _P64, _P64]
        L.ref_free.restype = None
        L.ref_free.argtypes = [C.c_void_p]
        _r = L
    return _r


# ---- oracle (C restatement) -----------------------------------------------------------

def bfs(row_offsets, column_indices, src, depth_limit=-1):
    """SimpleReferenceBfs restated: returns (labels, search_depth)."""
    n = row_offsets.size - 1
    labels = np.empty(n, dtype=np.int32)
    ci = column_indices if column_indices.size else np.zeros(1, np.int32)
    d = olib().oracle_bfs_limited(n, _p32(row_offsets), _p32(ci), int(src), int(depth_limit), _p32(labels))
    if d < 0:
        raise ValueError("oracle_bfs: bad arguments")
    return labels, int(d)


def check_predecessors(row_offsets, column_indices, ref_dist, preds):
    """Predecessor validity (test_bfs.cu:387-439): (-1, 0) when valid, else (node, reason)."""
    reason = C.c_int32(0)
    ci = column_indices if column_indices.size else np.zeros(1, np.int32)
    bad = olib().oracle_check_predecessors(row_offsets.size - 1, _p32(row_offsets), _p32(ci), _p32(ref_dist),
                                           _p32(preds), C.byref(reason))
    return int(bad), int(reason.value)


def visited_stats(row_offsets, labels):
    """(nodes_visited, edges_visited) as test_bfs.cu:359-367."""
    nv, ev = C.c_int64(0), C.c_int64(0)
    olib().oracle_visited_stats(row_offsets.size - 1, _p32(row_offsets), _p32(labels), C.byref(nv), C.byref(ev))
    return int(nv.value), int(ev.value)


def compare_labels(computed, reference):
    return int(olib().oracle_compare_labels(computed.size, _p32(computed), _p32(reference)))


def level_histogram(labels, max_levels=1 << 16):
    counts = np.zeros(max_levels, dtype=np.int64)
    n = olib().oracle_level_histogram(labels.size, _p32(labels), counts.ctypes.data_as(_P64), max_levels)
    return counts[:n]


# ---- the reference's own host code --------------------------------------------------------

def _take(L, ro_p, ci_p, n, m):
    n, m = int(n.value), int(m.value)
    ro = np.ctypeslib.as_array(ro_p, shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(ci_p, shape=(max(m, 1),))[:m].copy()
    L.ref_free(C.cast(ro_p, C.c_void_p))
    L.ref_free(C.cast(ci_p, C.c_void_p))
    return ro, ci


def ref_build(kind, *args):
    """Runs a reference builder; returns (row_offsets, column_indices)."""
    L = rlib()
    ro_p, ci_p = _P32(), _P32()
    n, m = C.c_int64(0), C.c_int64(0)
    rc = getattr(L, "ref_build_" + kind)(*args, C.byref(ro_p), C.byref(ci_p), C.byref(n), C.byref(m))
    if rc != 0:
        raise RuntimeError(f"reference builder {kind} failed")
    return _take(L, ro_p, ci_p, n, m)


def ref_read(kind, path, *args):
    """Runs a reference graph reader (market / dimacs / metis) on a file;
    returns (row_offsets, column_indices), or None when it reports an error."""
    L = rlib()
    ro_p, ci_p = _P32(), _P32()
    n, m = C.c_int64(0), C.c_int64(0)
    rc = getattr(L, "ref_read_" + kind)(os.fsencode(path), *args, C.byref(ro_p), C.byref(ci_p), C.byref(n),
                                        C.byref(m))
    if rc != 0:
        return None
    return _take(L, ro_p, ci_p, n, m)


def ref_bfs(row_offsets, column_indices, src):
    """The reference's SimpleReferenceBfs: (labels, search_depth, user_cpu_ms)."""
    L = rlib()
    n = row_offsets.size - 1
    labels = np.empty(n, dtype=np.int32)
    depth, ms = C.c_int64(0), C.c_double(0)
    ci = column_indices if column_indices.size else np.zeros(1, np.int32)
    L.ref_simple_bfs(n, column_indices.size, _p32(row_offsets), _p32(ci), int(src), _p32(labels), C.byref(depth),
                     C.byref(ms))
    return labels, int(depth.value), float(ms.value)


def bfs_many(row_offsets, column_indices, sources, threads=None):
    """Distances from each source, computed by independent serial searches in
    parallel threads (ctypes releases the GIL during each call): the
    reference's own SimpleReferenceBfs when its harness was built, else the C
    restatement.  Yields (source, labels, search_depth) in source order;
    search_depth = max label + 1 (what SimpleReferenceBfs reports)."""
    from concurrent.futures import ThreadPoolExecutor
    use_ref = have_ref()

    def one(s):
        if use_ref:
            labels = ref_bfs(row_offsets, column_indices, int(s))[0]
        else:
            labels = bfs(row_offsets, column_indices, int(s))[0]
        return int(s), labels, int(labels.max()) + 1

    threads = threads or max(1, min(len(sources), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=threads) as ex:
        yield from ex.map(one, list(sources))
