"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from back40computing_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(b40c_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "b40c_bfs_enact" in names and "b40c_bfs_problem_create" in names
    assert len(names) >= 20


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = ctypes.CDLL(N.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared but not exported"


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(N.SIGNATURES)


def test_no_device_reports_status():
    if N.device_count() > 0:
        pytest.skip("a GPU is present")
    import numpy as np
    ro = np.array([0, 1], np.int32)
    ci = np.array([0], np.int32)
    h = ctypes.c_void_p()
    rc = N.lib().b40c_bfs_problem_create(N.i32p(ro), N.i32p(ci), 1, 1, 0, 0, 0, ctypes.byref(h))
    assert rc == N.ERROR_NO_DEVICE
    assert "no CUDA device" in N.lib().b40c_last_error_string().decode()


def test_policy_validation_without_device():
    pol = N.Policy()
    assert N.lib().b40c_bfs_default_policy(0, ctypes.byref(pol)) == 0
    assert pol.threads == 256 and pol.chunk_edges == 2048
    assert N.lib().b40c_bfs_default_policy(9, ctypes.byref(pol)) == N.ERROR_INVALID_VALUE
