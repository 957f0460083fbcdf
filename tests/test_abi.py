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


def test_server_without_device_reports_status():
    if N.device_count() > 0:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert N.lib().b40c_server_create(0, None, ctypes.byref(h)) == N.ERROR_NO_DEVICE
    assert not h.value


def test_server_plan_bytes_arithmetic():
    """Admission's byte plan: the CSR, labels, masks, two vertex frontiers
    (1.3 n each), look-back slots and k label rows of the batch."""
    from back40computing_b200.server import BfsServer
    n, m = 1 << 20, 1 << 24
    b1, b2, b64 = (BfsServer.plan_bytes(n, m, k) for k in (1, 2, 64))
    assert b2 - b1 == 4 * n and b64 - b1 == 63 * 4 * n
    csr = 4 * (n + 1) + 4 * m
    # labels 4n, batch masks 24n + one label row 4n, two frontiers ~31n, hub pairs 8n,
    # unvisited lists 8n, slots ~m/256
    assert csr + 4 * n + 3 * 8 * n < b1 < csr + 88 * n + m // 8
    with pytest.raises(N.B40cError):
        BfsServer.plan_bytes(n, m, 65)


def test_unaligned_int32_arrays_are_rejected_before_any_device_call():
    """int32 arrays must start on a 4-byte boundary: the no-allocation search
    and problem creation refuse other addresses up front (no GPU touched)."""
    import numpy as np
    lib = N.lib()
    good, odd = ctypes.c_void_p(1 << 20), ctypes.c_void_p((1 << 20) + 2)
    for args in ((odd, good, good), (good, odd, good), (good, good, odd)):
        rc = lib.b40c_bfs_search_noalloc(args[0], args[1], 100, 400, 0, args[2], None)
        assert rc == N.ERROR_INVALID_VALUE
        assert "4-byte aligned" in lib.b40c_last_error_string().decode()
    raw = np.zeros(16, np.uint8)
    base = (-raw.ctypes.data) % 4
    ro = ctypes.cast(ctypes.c_void_p(raw.ctypes.data + base + 2),  # 2 bytes past a 4-byte boundary
                     ctypes.POINTER(ctypes.c_int32))
    h = ctypes.c_void_p()
    rc = lib.b40c_bfs_problem_create(ro, ro, 1, 0, 0, 1, 0, ctypes.byref(h))
    assert rc == N.ERROR_INVALID_VALUE and not h.value
