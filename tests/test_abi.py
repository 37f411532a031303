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


# Every function of the reference's C API (api/c/include/xkrt/xkrt.h:104-566), except the two it
# compiles out (#if 0: xkrt_driver_memory_device_info, xkrt_driver_device_cpuset).
REFERENCE_C_API = """
xkrt_init xkrt_deinit xkrt_reset xkrt_memory_register xkrt_memory_unregister xkrt_memory_register_async
xkrt_memory_unregister_async xkrt_file_read_async xkrt_file_write_async xkrt_memory_device_allocate
xkrt_memory_device_deallocate xkrt_memory_host_allocate xkrt_memory_host_deallocate xkrt_memory_unified_allocate
xkrt_memory_unified_deallocate xkrt_driver_get xkrt_device_get xkrt_device_driver_get xkrt_device_driver_id_get
xkrt_get_ndevices xkrt_get_ndevices_max xkrt_task_detachable_incr xkrt_task_detachable_decr xkrt_task_complete
xkrt_task_commit xkrt_task_enqueue xkrt_task_wait xkrt_task_args xkrt_task_accesses xkrt_task_access
xkrt_task_access_replica xkrt_task_current xkrt_task_spawn_generic xkrt_task_spawn_with_format
xkrt_task_spawn_with_format_with_accesses xkrt_task_spawn xkrt_task_kernel_launch xkrt_team_driver_device_get
xkrt_team_driver_get xkrt_team_driver_get_any xkrt_team_task_spawn xkrt_team_task_spawn_with_accesses
xkrt_task_format_put xkrt_task_format_set xkrt_driver_get_name xkrt_driver_get_ndevices_max xkrt_driver_init
xkrt_driver_finalize xkrt_driver_device_create xkrt_driver_device_init xkrt_driver_device_commit
xkrt_driver_device_destroy xkrt_driver_device_info xkrt_driver_memory_device_allocate
xkrt_driver_memory_device_deallocate xkrt_driver_memory_host_allocate xkrt_driver_memory_host_deallocate
xkrt_driver_memory_unified_allocate xkrt_driver_memory_unified_deallocate xkrt_driver_memory_host_register
xkrt_driver_memory_host_unregister xkrt_driver_memory_unified_advise_device xkrt_driver_memory_unified_advise_host
xkrt_driver_memory_unified_prefetch_device xkrt_driver_memory_unified_prefetch_host xkrt_driver_transfer_h2d
xkrt_driver_transfer_d2h xkrt_driver_transfer_d2d xkrt_driver_transfer_h2d_async xkrt_driver_transfer_d2h_async
xkrt_driver_transfer_d2d_async xkrt_device_kernel_launch xkrt_driver_kernel_launch xkrt_driver_queue_suggest
xkrt_driver_queue_create xkrt_driver_queue_delete xkrt_driver_module_load xkrt_driver_module_unload
xkrt_driver_module_get_fn xkrt_driver_power_start xkrt_driver_power_stop xkrt_logger_info xkrt_logger_debug
xkrt_logger_warn xkrt_logger_error xkrt_logger_fatal
""".split()


def test_reference_c_api_complete():
    """A program using any function of the reference's C API finds it declared and exported."""
    names = declared_symbols()
    assert set(REFERENCE_C_API) <= names, sorted(set(REFERENCE_C_API) - names)
    L = xk.lib()
    assert all(hasattr(L, n) for n in REFERENCE_C_API)


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
