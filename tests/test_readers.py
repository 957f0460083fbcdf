"""Graph file readers (MARKET / DIMACS / METIS) against an independent parse
and, where it was built, against the reference's own readers."""
import numpy as np
import pytest

import oracle
from back40computing_b200 import CsrGraph, BuildMarketGraph, BuildDimacsGraph, BuildMetisGraph, BuildRmatGraph

need_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built")


def _stable_csr(n, rows, cols):
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int32)
    order = np.argsort(rows, kind="stable")
    ro = np.zeros(n + 1, np.int32)
    np.add.at(ro, rows + 1, 1)
    return np.cumsum(ro).astype(np.int32), cols[order]


def _edges(seed, n=300, m=1500):
    rng = np.random.default_rng(seed)
    return rng.integers(1, n + 1, m), rng.integers(1, n + 1, m)


def _write_market(path, n, a, b, values=True):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n% a comment\n\n")
        f.write(f"{n} {n} {len(a)}\n")
        for x, y in zip(a, b):
            f.write(f"{x} {y} 0.5\n" if values else f"{x} {y}\n")


def _write_dimacs(path, n, u, v, header_first=True):
    with open(path, "w") as f:
        f.write("c a comment line\n")
        f.write(f"p sp {n} {len(u)}\n")
        for x, y in zip(u, v):
            f.write(f"a {x} {y} 7\n")


def _write_metis(path, n, adj, m_header, trailing_blank=False):
    with open(path, "w") as f:
        f.write("% comment before the header\n")
        f.write(f"{n} {m_header}\n")
        for v in range(n):
            if v == 3:
                f.write("% a comment between lines\n")
            f.write(" ".join(str(x + 1) for x in adj[v]) + "\n")
        if trailing_blank:
            f.write("\n\n")


def _read(fn, *args):
    g = CsrGraph()
    assert fn(*args[:1], g, *args[1:]) == 0
    return g


@pytest.mark.parametrize("undirected", [False, True])
def test_market_matches_independent_parse(tmp_path, undirected):
    n = 300
    a, b = _edges(1, n)
    p = tmp_path / "g.mtx"
    _write_market(p, n, a, b)
    g = _read(BuildMarketGraph, str(p), undirected)
    rows, cols = [], []
    for x, y in zip(a, b):  # first column is the column, second the row
        rows.append(y - 1)
        cols.append(x - 1)
        if undirected:
            rows.append(x - 1)
            cols.append(y - 1)
    ro, ci = _stable_csr(n, rows, cols)
    assert g.nodes == n and np.array_equal(g.row_offsets, ro) and np.array_equal(g.column_indices, ci)


@pytest.mark.parametrize("undirected", [False, True])
def test_dimacs_matches_independent_parse(tmp_path, undirected):
    n = 250
    u, v = _edges(2, n)
    p = tmp_path / "g.gr"
    _write_dimacs(p, n, u, v)
    g = _read(BuildDimacsGraph, str(p), undirected)
    rows, cols = [], []
    for x, y in zip(u, v):  # the reverse edge enters first
        if undirected:
            rows.append(y - 1)
            cols.append(x - 1)
        rows.append(x - 1)
        cols.append(y - 1)
    ro, ci = _stable_csr(n, rows, cols)
    assert np.array_equal(g.row_offsets, ro) and np.array_equal(g.column_indices, ci)


@pytest.mark.parametrize("listed", ["twice", "once"])
def test_metis_matches_independent_parse(tmp_path, listed):
    n = 200
    rng = np.random.default_rng(3)
    adj = [sorted(rng.choice(n, rng.integers(0, 6), replace=False).tolist()) for _ in range(n)]
    total = sum(len(a) for a in adj)
    if listed == "twice" and total % 2:
        adj[0].append(0)
        total += 1
    p = tmp_path / "g.graph"
    _write_metis(p, n, adj, total // 2 if listed == "twice" else total, trailing_blank=True)
    g = _read(BuildMetisGraph, str(p))
    ro = np.concatenate([[0], np.cumsum([len(a) for a in adj])]).astype(np.int32)
    ci = np.array([x for a in adj for x in a], np.int32)
    assert g.edges == total and np.array_equal(g.row_offsets, ro) and np.array_equal(g.column_indices, ci)


def test_rejects_malformed(tmp_path):
    bad = {
        "notsquare.mtx": "3 4 1\n1 1\n",
        "toomany.mtx": "3 3 1\n1 2\n2 3\n",
        "toofew.mtx": "3 3 3\n1 2\n",
        "range.mtx": "3 3 1\n1 4\n",
        "none.mtx": "% only a comment\n",
    }
    for name, text in bad.items():
        p = tmp_path / name
        p.write_text(text)
        assert BuildMarketGraph(str(p), CsrGraph(), False) == -1, name
    p = tmp_path / "few.gr"
    p.write_text("p sp 4 3\na 1 2 1\n")
    assert BuildDimacsGraph(str(p), CsrGraph(), False) == -1
    p = tmp_path / "range.gr"
    p.write_text("p sp 4 1\na 1 5 1\n")
    assert BuildDimacsGraph(str(p), CsrGraph(), False) == -1
    p = tmp_path / "many.graph"
    p.write_text("3 1\n2\n1\n3\n2\n")  # 4 ids for 2 * 1 expected
    assert BuildMetisGraph(str(p), CsrGraph()) == -1
    assert BuildMetisGraph(str(tmp_path / "missing.graph"), CsrGraph()) == -1


# ---- against the reference's readers --------------------------------------------------

def _rmat_edges():
    g = CsrGraph()
    BuildRmatGraph(1 << 10, 1 << 13, g, False, 0.57, 0.19, 0.19, seed=4)
    rows = np.repeat(np.arange(g.nodes), np.diff(g.row_offsets))
    return g.nodes, rows + 1, g.column_indices + 1, g


@need_ref
@pytest.mark.parametrize("undirected", [False, True])
def test_market_equals_reference_reader(tmp_path, undirected):
    n, r, c, _ = _rmat_edges()
    p = tmp_path / "r.mtx"
    _write_market(p, n, c, r)
    g = _read(BuildMarketGraph, str(p), undirected)
    want = oracle.ref_read("market", str(p), int(undirected))
    assert np.array_equal(g.row_offsets, want[0]) and np.array_equal(g.column_indices, want[1])


@need_ref
@pytest.mark.parametrize("undirected", [False, True])
@pytest.mark.parametrize("splice", [0, 3])
def test_dimacs_equals_reference_reader(tmp_path, undirected, splice):
    n, r, c, _ = _rmat_edges()
    if splice:
        # rows split round-robin over the splice files, each file in row order
        for i in range(splice):
            sel = (r - 1) % splice == i
            _write_dimacs(tmp_path / f"s.gr.{i}", n, r[sel], c[sel])
        path = str(tmp_path / "s.gr")
    else:
        path = str(tmp_path / "d.gr")
        _write_dimacs(path, n, r, c)
    g = _read(BuildDimacsGraph, path, undirected, splice)
    want = oracle.ref_read("dimacs", path, int(undirected), splice)
    assert np.array_equal(g.row_offsets, want[0]) and np.array_equal(g.column_indices, want[1])


@need_ref
def test_metis_equals_reference_reader(tmp_path):
    n, r, c, g0 = _rmat_edges()
    adj = [g0.column_indices[g0.row_offsets[v]:g0.row_offsets[v + 1]].tolist() for v in range(n)]
    total = g0.edges
    p = tmp_path / "r.graph"
    _write_metis(p, n, adj, total)  # header counts every listed id: the "once" form
    g = _read(BuildMetisGraph, str(p))
    want = oracle.ref_read("metis", str(p))
    assert np.array_equal(g.row_offsets, want[0]) and np.array_equal(g.column_indices, want[1])


@pytest.mark.gpu
def test_bfs_on_a_read_graph(tmp_path):
    from back40computing_b200 import CsrProblem, search, sample_sources, DIRECTION_OPTIMIZING
    n, r, c, _ = _rmat_edges()
    p = tmp_path / "r.mtx"
    _write_market(p, n, c, r)
    g = _read(BuildMarketGraph, str(p), True)
    prob = CsrProblem.from_graph(g)
    for s in sample_sources(g, 3, seed=1):
        got = search(prob, int(s), strategy=DIRECTION_OPTIMIZING)
        want, _ = oracle.bfs(g.row_offsets, g.column_indices, int(s))
        assert oracle.compare_labels(got, want) == -1
