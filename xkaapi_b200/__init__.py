"""xkaapi_b200 -- B200 (sm_100a) implementation of XKRT's dataflow hot path.

The product is the C-ABI shared library `libxkb200.so` (declared in include/xkrt_b200.h).
This module loads it with ctypes and exposes thin Python wrappers that take torch CUDA
tensors for device memory. There is no CPU fallback: if the library is missing or the GPU
is unreachable, calls raise XkbError.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxkb200.so")

XKB_OK = 0
XKB_EINVAL = -22
XKB_ENOMEM = -12
XKB_ERANGE = -34
XKB_ETIMEDOUT = -110
XKB_ENODEV = -19
XKB_ECUDA = -1000
F64, F32 = 0, 1
TASK_NOOP, TASK_HEAT_F64, TASK_HEAT_F32, TASK_AXPBY = 0, 1, 2, 3
FORM_PERSISTENT, FORM_PLAIN, FORM_GRAPH = 0, 1, 2
COPY_H2D, COPY_D2H, COPY_D2D = 0, 1, 2

_lib = None


class XkbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libxkb200 error {code}: {msg}")
        self.code = code


_c = ctypes
_i64, _dbl, _vp, _int = _c.c_int64, _c.c_double, _c.c_void_p, _c.c_int

class HeatCfg(ctypes.Structure):
    """xkb_heat_cfg_t: launch shape of the whole-step stencil kernel."""
    _fields_ = [("pf", ctypes.c_int), ("min_blocks", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("l2_prefetch_cols", ctypes.c_int), ("cols_per_strip", ctypes.c_int)]


class TaskGraph(ctypes.Structure):
    """xkb_task_graph_t: successor CSR in device memory."""
    _fields_ = [("ntasks", ctypes.c_uint64), ("nedges", ctypes.c_uint64), ("succ_ptr", ctypes.c_void_p),
                ("succ", ctypes.c_void_p), ("npred", ctypes.c_void_p)]


class ServerCfg(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("slots", ctypes.c_int), ("ctas_per_graph", ctypes.c_int),
                ("max_seconds", ctypes.c_double)]


class Request(ctypes.Structure):
    """xkb_request_t: one heat-diffusion request of a served stream."""
    _fields_ = [("arrival_s", ctypes.c_double), ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("ts", ctypes.c_int64),
                ("steps", ctypes.c_int32), ("f32", ctypes.c_int32), ("seed", ctypes.c_uint64), ("c", ctypes.c_double),
                ("result", ctypes.c_void_p), ("input", ctypes.c_void_p), ("start_s", ctypes.c_double),
                ("finish_s", ctypes.c_double)]


class PeriodicGraph(ctypes.Structure):
    """xkb_periodic_graph_t: one window's CSR plus its edges into the next window (device)."""
    _fields_ = [("period", ctypes.c_uint64), ("succ_ptr", ctypes.c_void_p), ("succ", ctypes.c_void_p),
                ("xsucc_ptr", ctypes.c_void_p), ("xsucc", ctypes.c_void_p), ("npred_first", ctypes.c_void_p),
                ("npred_next", ctypes.c_void_p)]


# name -> (restype, argtypes)
SIGNATURES = {
    "xkb_last_error": (_c.c_char_p, []),
    "xkb_version": (_c.c_char_p, []),
    "xkb_heat_tile": (_int, [_int, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _dbl, _vp]),
    "xkb_heat_step": (_int, [_int, _vp, _vp, _i64, _i64, _i64, _dbl, _vp]),
    "xkb_heat_step_cfg": (_int, [_int, _vp, _vp, _i64, _i64, _i64, _dbl, ctypes.POINTER(HeatCfg), _vp]),
    "xkb_heat_norms": (_int, [_int, _vp, _vp, _i64, _i64, _i64, _dbl, _vp, _vp]),
    "xkb_planner_set_device_budget": (_int, [_vp, ctypes.c_uint64]),
    "xkb_planner_allocation_offsets": (_int, [_vp, _vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "xkb_planner_eviction_stats": (_int, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "xkb_planner_set_writeback_coherent": (_int, [_vp, _int]),
    "xkb_axpby": (_int, [_i64, _dbl, _vp, _dbl, _vp, _vp]),
    "xkb_sched_create": (_int, [ctypes.POINTER(_vp), _vp]),
    "xkb_sched_destroy": (_int, [_vp]),
    "xkb_sched_set_tasks": (_int, [_vp, _vp, ctypes.c_size_t]),
    "xkb_sched_set_timeout": (_int, [_vp, _dbl]),
    "xkb_sched_set_grid": (_int, [_vp, _int]),
    "xkb_sched_set_team": (_int, [_vp, _int]),
    "xkb_sched_set_prefetch": (_int, [_vp, _int]),
    "xkb_sched_set_staging": (_int, [_vp, _int]),
    "xkb_sched_run": (_int, [_vp, ctypes.POINTER(TaskGraph), _int]),
    "xkb_sched_wait": (_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "xkb_sched_kernel_ms": (_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "xkb_sched_run_noalloc": (_int, [_vp, ctypes.POINTER(TaskGraph), _int, _dbl, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    "xkb_planner_create": (_int, [ctypes.POINTER(_vp)]),
    "xkb_planner_destroy": (_int, [_vp]),
    "xkb_planner_create_resident": (_int, [ctypes.POINTER(_vp)]),
    "xkb_planner_add_region": (_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]),
    "xkb_planner_flush_to_host": (_int, [_vp]),
    "xkb_planner_invalidate": (_int, [_vp]),
    "xkb_planner_replace_regions": (_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]),
    "xkb_planner_register": (_int, [_vp, ctypes.c_uint64, ctypes.c_uint64]),
    "xkb_planner_unregister": (_int, [_vp, ctypes.c_uint64, ctypes.c_uint64]),
    "xkb_planner_fetch": (_int, [_vp, _vp, ctypes.c_uint32, _int, _vp]),
    "xkb_planner_plan": (_int, [_vp, _vp, ctypes.c_size_t, _int, _vp]),
    "xkb_planner_copies": (_int, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), _int]),
    "xkb_planner_allocations": (_int, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "xkb_plan_execute": (_int, [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]),
    "xkb_diffusion_views": (_int, [_int, _vp, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _dbl]),
    "xkb_server_create": (_int, [ctypes.POINTER(_vp), ctypes.POINTER(ServerCfg)]),
    "xkb_server_destroy": (_int, [_vp]),
    "xkb_server_run": (_int, [_vp, ctypes.POINTER(Request), ctypes.c_size_t]),
    "xkb_resolver_create": (_int, [ctypes.POINTER(_vp), _vp]),
    "xkb_resolver_periodic": (_int, [_vp, ctypes.c_uint64, ctypes.POINTER(PeriodicGraph)]),
    "xkb_sched_run_periodic": (_int, [_vp, ctypes.POINTER(PeriodicGraph), ctypes.c_uint32, ctypes.c_uint32]),
    "xkb_resolver_destroy": (_int, [_vp]),
    "xkb_handle_map_create": (_int, [ctypes.POINTER(_vp)]),
    "xkb_handle_map_destroy": (_int, [_vp]),
    "xkb_handle_map_expand": (_int, [_vp, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "xkb_resolver_add": (_int, [_vp, _vp, ctypes.c_size_t]),
    "xkb_resolver_reset": (_int, [_vp]),
    "xkb_resolver_graph": (_int, [_vp, ctypes.POINTER(TaskGraph)]),
    "xkb_resolver_edges": (_int, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "xkb_resolver_stats": (_int, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                  ctypes.POINTER(ctypes.c_double)]),
    "xkb_resolver_timing": (_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]),
}


def lib():
    """Load libxkb200.so (built in-tree by xkaapi_b200/build.py). Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise XkbError(XKB_ENODEV, f"{LIB_PATH} is not built (run: python -m xkaapi_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def check(rc):
    if rc != XKB_OK:
        raise XkbError(rc, lib().xkb_last_error().decode())
    return rc


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _dtype_code(t):
    import torch
    if t.dtype == torch.float64:
        return F64
    if t.dtype == torch.float32:
        return F32
    raise XkbError(XKB_EINVAL, f"unsupported grid dtype {t.dtype}")


def heat_tile(src, dst, nx, ny, ld, tile_x, tile_y, tsx, tsy, c, stream=None):
    """One heat tile task on whole resident grids (torch CUDA tensors, column-major with ld)."""
    return check(lib().xkb_heat_tile(_dtype_code(src), src.data_ptr(), dst.data_ptr(), ld, nx, ny,
                                     tile_x, tile_y, tsx, tsy, c, _stream(stream)))


def heat_step(src, dst, nx, ny, ld, c, stream=None, cfg=None):
    """One whole Jacobi step over the grid in one launch (cfg: HeatCfg or None for the default)."""
    if cfg is None:
        return check(lib().xkb_heat_step(_dtype_code(src), src.data_ptr(), dst.data_ptr(), ld, nx, ny, c,
                                         _stream(stream)))
    return check(lib().xkb_heat_step_cfg(_dtype_code(src), src.data_ptr(), dst.data_ptr(), ld, nx, ny, c,
                                         ctypes.byref(cfg), _stream(stream)))


def heat_norms(src, dst, nx, ny, ld, c, stream=None):
    """FP64 checks of the step src -> dst (torch CUDA grids of either storage type): the largest
    |dst| on the boundary, the interior L2 norm, the step's residual max |dst - update(src)| and
    the largest interior |dst| (xkb_heat_norms)."""
    import torch
    out = torch.zeros(4, dtype=torch.float64, device=src.device)
    torch.cuda.current_stream().synchronize()        # the zeros are in place before the library's stream clears them
    check(lib().xkb_heat_norms(_dtype_code(src), src.data_ptr(), dst.data_ptr(), ld, nx, ny, c, out.data_ptr(), _stream(stream)))
    getattr(stream, "synchronize", torch.cuda.synchronize)()
    o = out.cpu().tolist()
    return {"boundary_max_abs": o[0], "l2_norm": o[1] ** 0.5, "residual_max_abs": o[2], "interior_max_abs": o[3]}


def axpby(a, x, b, y, stream=None):
    """y = a*x + b*y (FP64 torch CUDA tensors)."""
    return check(lib().xkb_axpby(x.numel(), a, x.data_ptr(), b, y.data_ptr(), _stream(stream)))


class Resolver:
    """Batched GPU dependency resolver (xkb_resolver_t). Feed access records (numpy structured
    array with the 64-byte xkb_access_rec_t layout) in spawn order; read back unique edges or
    the device successor graph."""

    def __init__(self, stream=None):
        self._h = ctypes.c_void_p()
        check(lib().xkb_resolver_create(ctypes.byref(self._h), _stream(stream) if stream is not None else None))

    def add(self, recs):
        import numpy as np
        recs = np.ascontiguousarray(recs)
        assert recs.dtype.itemsize == 64
        check(lib().xkb_resolver_add(self._h, recs.ctypes.data, len(recs)))

    def edges(self):
        import numpy as np
        n = ctypes.c_size_t()
        rc = lib().xkb_resolver_edges(self._h, None, 0, ctypes.byref(n))
        if rc not in (XKB_OK, XKB_ERANGE):
            check(rc)
        out = np.zeros((n.value, 2), dtype=np.uint32)
        check(lib().xkb_resolver_edges(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def graph(self):
        g = TaskGraph()
        check(lib().xkb_resolver_graph(self._h, ctypes.byref(g)))
        return g

    def reset(self):
        """Forget every task and edge; keep the working buffers."""
        check(lib().xkb_resolver_reset(self._h))

    def periodic(self, period):
        g = PeriodicGraph()
        check(lib().xkb_resolver_periodic(self._h, period, ctypes.byref(g)))
        return g

    def stats(self):
        nt, ne, ms = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double()
        check(lib().xkb_resolver_stats(self._h, ctypes.byref(nt), ctypes.byref(ne), ctypes.byref(ms)))
        return nt.value, ne.value, ms.value

    def timing(self):
        """(ops_ms, compress_ms, batch_ms) of the last batch."""
        o, c, b = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().xkb_resolver_timing(self._h, ctypes.byref(o), ctypes.byref(c), ctypes.byref(b)))
        return o.value, c.value, b.value

    def close(self):
        if self._h:
            lib().xkb_resolver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def task_desc_dtype():
    """numpy dtype of xkb_task_desc_t (64 bytes); heat and axpby views share the union bytes."""
    import numpy as np
    return np.dtype({"names": ["kind", "flags", "src", "dst", "ld", "nx", "ny", "x0", "x1", "y0", "y1", "c"],
                     "formats": ["<u4", "<u4", "<u8", "<u8", "<i8", "<i4", "<i4", "<i4", "<i4", "<i4", "<i4", "<f8"],
                     "offsets": [0, 4, 8, 16, 24, 32, 36, 40, 44, 48, 52, 56], "itemsize": 64})


def axpby_desc_dtype():
    import numpy as np
    return np.dtype({"names": ["kind", "flags", "x", "y", "lo", "hi", "a", "b"],
                     "formats": ["<u4", "<u4", "<u8", "<u8", "<i8", "<i8", "<f8", "<f8"],
                     "offsets": [0, 4, 8, 16, 24, 32, 40, 48], "itemsize": 64})


class Scheduler:
    """Device scheduler (xkb_sched_t): runs a resolved task graph in one of three forms."""

    def __init__(self, stream=None):
        self._h = ctypes.c_void_p()
        check(lib().xkb_sched_create(ctypes.byref(self._h), _stream(stream) if stream is not None else None))

    def set_tasks(self, descs):
        import numpy as np
        descs = np.ascontiguousarray(descs)
        assert descs.dtype.itemsize == 64
        check(lib().xkb_sched_set_tasks(self._h, descs.ctypes.data, len(descs)))

    def set_timeout(self, seconds):
        check(lib().xkb_sched_set_timeout(self._h, seconds))

    def set_grid(self, ctas):
        check(lib().xkb_sched_set_grid(self._h, ctas))

    def set_team(self, warps_per_task):
        check(lib().xkb_sched_set_team(self._h, warps_per_task))

    def set_prefetch(self, columns):
        check(lib().xkb_sched_set_prefetch(self._h, columns))

    def set_staging(self, bulk):
        """Heat tile body of the persistent kernel: False = register body (default), True = bulk-staged."""
        check(lib().xkb_sched_set_staging(self._h, 1 if bulk else 0))

    def run(self, graph, form=FORM_PERSISTENT):
        check(lib().xkb_sched_run(self._h, ctypes.byref(graph), form))

    def run_periodic(self, graph, repeats, tail=None):
        check(lib().xkb_sched_run_periodic(self._h, ctypes.byref(graph), repeats,
                                           graph.period if tail is None else tail))

    def wait(self):
        n = ctypes.c_uint64()
        check(lib().xkb_sched_wait(self._h, ctypes.byref(n)))
        return n.value

    def kernel_ms(self):
        ms = ctypes.c_double()
        check(lib().xkb_sched_kernel_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self._h:
            lib().xkb_sched_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from .heat import heat_task_descs, heat_access_records  # noqa: E402,F401


class Planner:
    """Coherency/transfer planner (xkb_planner_t, host code: no GPU needed). Copies come back as
    an (n, 14) int64 array: task, access, kind, src_dev, src_alloc, src_off, src_ld, dst_dev,
    dst_alloc, dst_off, dst_ld, m, n, sizeof."""

    def __init__(self, resident=False, budget=0):
        self._h = ctypes.c_void_p()
        if resident:
            check(lib().xkb_planner_create_resident(ctypes.byref(self._h)))
        else:
            check(lib().xkb_planner_create(ctypes.byref(self._h)))
            if budget:
                check(lib().xkb_planner_set_device_budget(self._h, budget))

    def offsets(self):
        """(offset, live) of every allocation in the device budget."""
        import numpy as np
        n = ctypes.c_size_t()
        check(lib().xkb_planner_allocation_offsets(self._h, None, None, 0, ctypes.byref(n)))
        out, live = np.zeros(n.value, dtype=np.int64), np.zeros(n.value, dtype=np.uint8)
        check(lib().xkb_planner_allocation_offsets(self._h, out.ctypes.data, live.ctypes.data, n.value, ctypes.byref(n)))
        return out, live.astype(bool)

    def eviction_stats(self):
        e, w = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().xkb_planner_eviction_stats(self._h, ctypes.byref(e), ctypes.byref(w)))
        return e.value, w.value

    def add_region(self, base, size):
        r = ctypes.c_int32()
        check(lib().xkb_planner_add_region(self._h, base, size, ctypes.byref(r)))
        return r.value

    def replace_regions(self, base, size):
        """Resident mode: the regions inside [base, base + size) become one region (new ordinal)."""
        r = ctypes.c_int32()
        check(lib().xkb_planner_replace_regions(self._h, base, size, ctypes.byref(r)))
        return r.value

    def flush_to_host(self):
        check(lib().xkb_planner_flush_to_host(self._h))

    def register(self, ptr, size):
        """Host memory [ptr, ptr + size) registered (registration-overflow protection)."""
        check(lib().xkb_planner_register(self._h, ptr, size))

    def unregister(self, ptr, size):
        check(lib().xkb_planner_unregister(self._h, ptr, size))

    def invalidate(self):
        """Forget every device copy (the host's is the only coherent one again)."""
        check(lib().xkb_planner_invalidate(self._h))

    def plan(self, recs, device=1):
        import numpy as np
        recs = np.ascontiguousarray(recs)
        views = np.zeros((len(recs), 3), dtype=np.int64)
        check(lib().xkb_planner_plan(self._h, recs.ctypes.data, len(recs), device, views.ctypes.data))
        return views

    def fetch(self, rec, access_index, device=1):
        import numpy as np
        rec = np.ascontiguousarray(rec).reshape(1)
        v = np.zeros(3, dtype=np.int64)
        check(lib().xkb_planner_fetch(self._h, rec.ctypes.data, access_index, device, v.ctypes.data))
        return v

    def copies(self, take=False):
        import numpy as np
        n = ctypes.c_size_t()
        check(lib().xkb_planner_copies(self._h, None, 0, ctypes.byref(n), 0))
        out = np.zeros((n.value, 14), dtype=np.int64)
        check(lib().xkb_planner_copies(self._h, out.ctypes.data, n.value, ctypes.byref(n), 1 if take else 0))
        return out

    def allocations(self):
        import numpy as np
        n = ctypes.c_size_t()
        check(lib().xkb_planner_allocations(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.uint64)
        check(lib().xkb_planner_allocations(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def close(self):
        if self._h:
            lib().xkb_planner_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HandleMap:
    """xkb_handle_map_t (host code: no GPU needed): expands access records holding
    concurrent-mode handle accesses (record field `reserved` >> 8 == 4) into a stream the
    resolver takes -- the reference handle map's extra writer tasks inserted, later tasks
    renumbered, concurrent writes resolved as reads. Keeps its state across calls."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        check(lib().xkb_handle_map_create(ctypes.byref(self._h)))

    def expand(self, recs):
        import numpy as np
        recs = np.ascontiguousarray(recs)
        out = np.zeros(2 * len(recs), dtype=recs.dtype)
        n = ctypes.c_size_t()
        check(lib().xkb_handle_map_expand(self._h, recs.ctypes.data, len(recs), out.ctypes.data, len(out), ctypes.byref(n)))
        return out[:n.value]

    def close(self):
        if self._h:
            lib().xkb_handle_map_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_execute(copies, alloc_ptrs, stream=None):
    """Execute planned copies ((n, 14) int64 array) with the given allocation base pointers."""
    import numpy as np
    copies = np.ascontiguousarray(copies, dtype=np.int64)
    ptrs = (ctypes.c_void_p * max(1, len(alloc_ptrs)))(*alloc_ptrs)
    check(lib().xkb_plan_execute(copies.ctypes.data, len(copies), ptrs, len(alloc_ptrs), _stream(stream)))


class Server:
    """Serving loop (xkb_server_t): continuous admission of heat graphs under an HBM budget."""

    def __init__(self, budget_bytes, slots=8, ctas_per_graph=0, max_seconds=600.0):
        self._h = ctypes.c_void_p()
        cfg = ServerCfg(int(budget_bytes), slots, ctas_per_graph, max_seconds)
        check(lib().xkb_server_create(ctypes.byref(self._h), ctypes.byref(cfg)))

    def run(self, reqs):
        """reqs: a ctypes array of Request (filled in place with start_s / finish_s)."""
        check(lib().xkb_server_run(self._h, reqs, len(reqs)))
        return reqs

    def close(self):
        if self._h:
            lib().xkb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
