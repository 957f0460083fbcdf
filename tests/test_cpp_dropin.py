"""The C++ drop-in headers (include/b40c/...): a caller written against the
reference's API compiles unchanged and links to libb40c_bfs.so; the libc
rand() builders reproduce the reference builders' graphs exactly after the
same srand() seed; on a GPU every enactor validates against a CPU BFS."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from back40computing_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
LIBDIR = os.path.join(ROOT, "back40computing_b200", "lib")


def _compile(name, out_dir):
    exe = os.path.join(out_dir, name)
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), "-I" + CUDA_INC,
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o", exe, "-L" + LIBDIR, "-lb40c_bfs",
           "-Wl,-rpath," + LIBDIR]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.fixture(scope="module")
def exes(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cpp"))
    return {n: _compile(n, d) for n in ("test_bfs_dropin", "builder_dump")}


def _dump(exe, tmp, seed, *args):
    out = os.path.join(tmp, "g.bin")
    subprocess.run([exe, out, str(seed), *map(str, args)], check=True, capture_output=True)
    raw = open(out, "rb").read()
    n, m = np.frombuffer(raw[:16], dtype=np.int64)
    ro = np.frombuffer(raw[16:16 + 4 * (n + 1)], dtype=np.int32)
    ci = np.frombuffer(raw[16 + 4 * (n + 1):], dtype=np.int32)
    assert ci.size == m
    return ro, ci


def test_headers_compile_and_link(exes):
    assert os.access(exes["test_bfs_dropin"], os.X_OK)


def test_lattices_match_native_builder(exes, tmp_path):
    from back40computing_b200 import CsrGraph, BuildGrid2dGraph, BuildGrid3dGraph
    for kind, w, fn in (("grid2d", 37, BuildGrid2dGraph), ("grid3d", 9, BuildGrid3dGraph), ("grid2d", 1, BuildGrid2dGraph)):
        ro, ci = _dump(exes["builder_dump"], str(tmp_path), 0, kind, w)
        g = CsrGraph()
        fn(w, g)
        assert np.array_equal(ro, g.row_offsets) and np.array_equal(ci, g.column_indices)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built")
@pytest.mark.parametrize("seed", [0, 7])
@pytest.mark.parametrize("kind,args,ref_args", [
    ("rmat", (2048, 16384, 1), (2048, 16384, 1, 0.57, 0.19, 0.19)),
    ("rmat", (1024, 5000, 0), (1024, 5000, 0, 0.57, 0.19, 0.19)),
    ("random", (3000, 9000, 1), (3000, 9000, 1)),
    ("rr", (2500, 5), (2500, 5)),
])
def test_rand_builders_match_reference_exactly(exes, tmp_path, kind, args, ref_args, seed):
    ro, ci = _dump(exes["builder_dump"], str(tmp_path), seed, kind, *args)
    rro, rci = oracle.ref_build(kind, *ref_args, seed)
    assert np.array_equal(ro, rro) and np.array_equal(ci, rci)


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    ["grid2d", "60"], ["grid3d", "14", "--mark-pred"], ["rmat", "8192", "65536"], ["rmat", "8192", "65536", "--mark-pred"],
    ["random", "5000", "20000"], ["rr", "6000", "4"], ["grid2d", "40", "--instrumented"],
])
def test_dropin_driver_validates_on_gpu(exes, args):
    r = subprocess.run([exes["test_bfs_dropin"], *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert r.stdout.count("CORRECT") >= 6 and "INCORRECT" not in r.stdout


def test_file_readers_through_cpp_headers(exes, tmp_path):
    """BuildMarketGraph / BuildDimacsGraph / BuildMetisGraph from the C++
    headers give the graphs the Python readers give."""
    from back40computing_b200 import CsrGraph, BuildMarketGraph, BuildDimacsGraph, BuildMetisGraph
    rng = np.random.default_rng(5)
    n, m = 120, 700
    a, b = rng.integers(1, n + 1, m), rng.integers(1, n + 1, m)
    mtx = tmp_path / "g.mtx"
    mtx.write_text(f"%%MatrixMarket matrix coordinate pattern general\n{n} {n} {m}\n" +
                   "".join(f"{x} {y}\n" for x, y in zip(a, b)))
    gr = tmp_path / "g.gr"
    gr.write_text(f"p sp {n} {m}\n" + "".join(f"a {x} {y} 1\n" for x, y in zip(a, b)))
    met = tmp_path / "g.graph"
    adj = [[] for _ in range(n)]
    for x, y in zip(a, b):
        adj[x - 1].append(y)
    met.write_text(f"{n} {m}\n" + "".join(" ".join(map(str, row)) + "\n" for row in adj))
    cases = [(("market", mtx, 1), lambda g: BuildMarketGraph(str(mtx), g, True)),
             (("dimacs", gr, 0, 0), lambda g: BuildDimacsGraph(str(gr), g, False)),
             (("metis", met), lambda g: BuildMetisGraph(str(met), g))]
    for args, fn in cases:
        ro, ci = _dump(exes["builder_dump"], str(tmp_path), 0, *args)
        g = CsrGraph()
        assert fn(g) == 0
        assert np.array_equal(ro, g.row_offsets) and np.array_equal(ci, g.column_indices), args[0]


REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "test_bfs_dropin")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="reference driver not built (oracle/build_dropin.sh)")
@pytest.mark.parametrize("args,strategies", [
    (["grid2d", "300", "--src=0"], 5),
    (["grid3d", "40", "--src=0", "--mark-pred"], 4),
    (["rmat", "65536", "1048576", "--undirected", "--src=randomize", "--i=2"], 4),
    (["rmat", "65536", "1048576", "--undirected", "--src=randomize", "--mark-pred"], 4),
    (["rmat", "32768", "262144", "--undirected", "--src=randomize", "--stream-from-host"], 5),
    (["g500", "32768", "--src=randomize"], 5),
    (["random", "20000", "100000", "--undirected", "--src=randomize"], 4),
    (["rr", "20000", "6", "--src=randomize", "--queue-sizing=2.0"], 4),
])
def test_reference_driver_unchanged_validates_on_gpu(args, strategies):
    """The reference's own driver (test/bfs/test_bfs.cu: RunTests and main),
    compiled unchanged against include/ by oracle/build_dropin.sh, runs every
    enactor it knows (expand-contract, contract-expand, two-phase, hybrid and,
    on one GPU, the multi-GPU one) and checks each against its own CPU BFS:
    every GPU search prints CORRECT.  Covers 64-bit vertex ids (g500) and the
    zero-copy --stream-from-host mode."""
    strat = ",".join(str(s) for s in range(strategies))
    r = subprocess.run([REF_DRIVER, *args, f"--strategy={strat}"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    iters = 2 if "--i=2" in args else 1
    assert "INCORRECT" not in r.stdout, r.stdout[-3000:]
    assert r.stdout.count("CORRECT") == strategies * iters, r.stdout[-3000:]
