"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import os
import re

import xkaapi_b200 as xk

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(REPO, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"XKB_API\s+[\w\s\*]+?\b(xk\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_all_declared_symbols():
    L = xk.lib()
    names = declared_symbols()
    assert names, "no XKB_API declarations found"
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_python_signatures_cover_header():
    # the xkb_* library API is bound in Python; the xkrt_* C API is for C programs
    xkb = {n for n in declared_symbols() if n.startswith("xkb_")}
    assert xkb - set(xk.SIGNATURES) <= {"xkb_task_format_builtin", "xkb_runtime_status", "xkb_runtime_stream",
                                        "xkb_runtime_last_wait", "xkb_runtime_last_wait_times",
                                        "xkb_runtime_last_wait_bytes"}, xkb - set(xk.SIGNATURES)


def test_c_api_symbols_exported():
    names = {n for n in declared_symbols() if n.startswith("xkrt_")}
    assert {"xkrt_init", "xkrt_task_spawn_generic", "xkrt_task_wait", "xkrt_task_format_put"} <= names
    L = xk.lib()
    assert all(hasattr(L, n) for n in names)


def test_version_reports_sm100a():
    assert b"sm_100a" in xk.lib().xkb_version()


def test_bad_arguments_rejected_without_gpu():
    L = xk.lib()
    # dtype out of range and src == dst are rejected on the host before any CUDA call
    assert L.xkb_heat_step(7, 16, 32, 8, 8, 8, 0.2, None) == xk.XKB_EINVAL
    assert L.xkb_heat_step(xk.F64, 16, 16, 8, 8, 8, 0.2, None) == xk.XKB_EINVAL
    assert b"distinct" in L.xkb_last_error()
    assert L.xkb_axpby(-1, 1.0, None, 1.0, None, None) == xk.XKB_EINVAL


def test_access_record_is_64_bytes():
    import streams
    assert streams.REC.itemsize == 64
