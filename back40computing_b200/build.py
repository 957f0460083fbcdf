"""Builds the native pieces in-tree.

* ``back40computing_b200/lib/libb40c_bfs.so`` -- the product: sm_100a kernels,
  the host runtime and the C ABI declared in ``include/b40c_bfs.h`` (nvcc,
  ``-gencode arch=compute_100a,code=sm_100a``).
* ``oracle/liboracle.so`` -- the CPU oracle (test infrastructure, gcc).
* ``oracle/_ref/libb40c_ref.so`` -- the reference's own host code, and
  ``oracle/_ref/test_bfs_dropin`` -- the reference's BFS driver compiled
  unchanged against ``include/``, when a reference tree is given
  (``$B40C_REFERENCE_TREE`` or ``--reference <tree>``; ``oracle/build_ref.sh``,
  ``oracle/build_dropin.sh``; test infrastructure).

Run ``python -m back40computing_b200.build [--force] [--reference <tree>]``
(or call :func:`build_all`).
Sources are rebuilt only when newer than their outputs.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")
ORACLE = os.path.join(ROOT, "oracle")
LIB = os.path.join(LIBDIR, "libb40c_bfs.so")
ORACLE_LIB = os.path.join(ORACLE, "liboracle.so")
REF_LIB = os.path.join(ORACLE, "_ref", "libb40c_ref.so")
DROPIN_EXE = os.path.join(ORACLE, "_ref", "test_bfs_dropin")
# the reference tree (read only) for the test harnesses under oracle/_ref; unset: not built
REFERENCE_TREE = os.environ.get("B40C_REFERENCE_TREE")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], cwd: str | None = None) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def build_library(force: bool = False, verbose_ptxas: bool = False) -> str:
    deps = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if not force and not _newer(LIB, deps):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
    cmds, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", *common, "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmds.append(["g++", "-O3", "-std=c++17", "-fPIC", "-pthread", "-I" + INCLUDE, "-I" + CSRC,
                     "-I" + os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj])
        objs.append(obj)
    # translation units compile independently: one compiler process per core
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, cmds))
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lpthread"])
    os.replace(tmp, LIB)
    shutil.rmtree(objdir, ignore_errors=True)
    return LIB


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ORACLE, "bfs_oracle.c")
    if force or _newer(ORACLE_LIB, [src]):
        tmp = ORACLE_LIB + ".tmp"
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=c99", src, "-o", tmp])
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_reference(force: bool = False, tree: str | None = None) -> str | None:
    """Builds oracle/_ref (the reference's own CPU BFS harness and its BFS
    driver compiled against include/) from the reference tree `tree` (default:
    $B40C_REFERENCE_TREE) when it is present; test infrastructure only."""
    tree = tree or REFERENCE_TREE
    if not tree or not os.path.isfile(os.path.join(tree, "test", "bfs", "test_bfs.cu")):
        return REF_LIB if os.path.exists(REF_LIB) else None
    deps = [os.path.join(ORACLE, "ref_harness.cpp"), os.path.join(ORACLE, "build_ref.sh")]
    if force or _newer(REF_LIB, deps):
        _run(["bash", os.path.join(ORACLE, "build_ref.sh"), tree])
    deps = [LIB, os.path.join(ORACLE, "build_dropin.sh")] + glob.glob(os.path.join(INCLUDE, "**", "*"), recursive=True)
    if force or _newer(DROPIN_EXE, [d for d in deps if os.path.isfile(d)]):
        _run(["bash", os.path.join(ORACLE, "build_dropin.sh"), tree])
    return REF_LIB


def build_all(force: bool = False, reference_tree: str | None = None) -> None:
    build_library(force)
    build_oracle(force)
    build_reference(force, reference_tree)


if __name__ == "__main__":
    tree = sys.argv[sys.argv.index("--reference") + 1] if "--reference" in sys.argv else None
    build_all(force="--force" in sys.argv, reference_tree=tree)
