"""The persistent run that allocates nothing (xkb_sched_run_noalloc), called through the C ABI.

It is meant for callers that cannot allocate device memory while they run a graph -- a runtime
that has reserved most of the GPU's memory for its own allocator, a serving loop with fixed
memory pools, a loop where cudaMalloc would synchronise the device -- so it keeps its counters
and queue in a fixed array of the library. This test checks that it computes exactly what the
allocating scheduler computes, on two calls in a row (the second call finds the array holding
the first call's contents). This file is collected last so a failure here leaves the rest of
the suite already run."""
import ctypes

import numpy as np
import pytest

import kernels_oracle as O
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu


def _setup_call(torch):
    """The set-up call the header asks for: an empty graph, once per device, before the caller
    reserves memory or captures a stream. It loads the library's array and kernels."""
    empty = xk.TaskGraph(0, 0, 0, 0, 0)
    rc = xk.lib().xkb_sched_run_noalloc(None, ctypes.byref(empty), 2, 1.0, torch.cuda.current_stream().cuda_stream, None)
    xk.check(rc)


def test_noalloc_run_matches_allocating_scheduler_twice(torch_cuda):
    torch = torch_cuda
    _setup_call(torch)
    nx = ny = 256
    ts, steps, c = 64, 6, 0.2
    g = O.heat_init(nx, ny, seed=5)
    a1, b1 = torch.from_numpy(g).cuda(), torch.from_numpy(g).cuda()     # allocating scheduler
    a2, b2 = torch.from_numpy(g).cuda(), torch.from_numpy(g).cuda()     # no-allocation entry point
    res = xk.Resolver()
    res.add(xk.heat_access_records(nx, ny, ts, ts, 0, steps, a1.data_ptr(), b1.data_ptr()))
    graph = res.graph()                    # same dependency structure for any pair of grids
    d1 = xk.heat_task_descs((a1.data_ptr(), b1.data_ptr()), nx, ny, nx, ts, ts, steps, c)
    d2 = xk.heat_task_descs((a2.data_ptr(), b2.data_ptr()), nx, ny, nx, ts, ts, steps, c)
    d2_dev = torch.from_numpy(d2.view(np.uint8).copy()).cuda()          # device array of descriptors
    sch = xk.Scheduler()
    sch.set_tasks(d1)
    stream = torch.cuda.current_stream()
    for call in range(2):
        sch.run(graph)
        assert sch.wait() == len(d1)
        executed = ctypes.c_uint64()
        rc = xk.lib().xkb_sched_run_noalloc(d2_dev.data_ptr(), ctypes.byref(graph), 2, 10.0, stream.cuda_stream,
                                            ctypes.byref(executed))
        xk.check(rc)
        assert executed.value == len(d2)
        torch.cuda.synchronize()
        out1 = (a1 if steps % 2 == 0 else b1).cpu().numpy()
        out2 = (a2 if steps % 2 == 0 else b2).cpu().numpy()
        np.testing.assert_array_equal(out2, out1)                          # bit-exact, as elsewhere
        np.testing.assert_array_equal(out1, O.heat_run(g, nx, ny, steps * (call + 1), c))


def test_noalloc_rejects_graphs_beyond_capacity(torch_cuda):
    torch = torch_cuda
    graph = xk.TaskGraph((1 << 20) + 1, 0, 16, 16, 16)      # checked on the host before any device access
    rc = xk.lib().xkb_sched_run_noalloc(16, ctypes.byref(graph), 2, 1.0, None, None)
    assert rc == xk.XKB_ERANGE
    assert b"fixed capacity" in xk.lib().xkb_last_error()


def test_noalloc_rejects_bad_descriptors_and_runs_nothing(torch_cuda):
    """Descriptors are checked on the device before the run: an unknown kind or a reversed axpby
    range returns XKB_EINVAL naming the first bad task, and no task runs. (Both forms would be
    no-ops in the tile bodies, so the check is shown without any risky memory access.)"""
    torch = torch_cuda
    _setup_call(torch)
    nx = ny = 128
    g = O.heat_init(nx, ny, seed=9)
    a, b = torch.from_numpy(g).cuda(), torch.from_numpy(g).cuda()
    res = xk.Resolver()
    res.add(xk.heat_access_records(nx, ny, 64, 64, 0, 2, a.data_ptr(), b.data_ptr()))
    graph = res.graph()
    d = xk.heat_task_descs((a.data_ptr(), b.data_ptr()), nx, ny, nx, 64, 64, 2, 0.2)
    stream = torch.cuda.current_stream().cuda_stream
    for bad_index, corrupt in ((5, "kind"), (2, "range")):
        bad = d.copy()
        raw = bad.view(np.uint8).reshape(len(bad), -1)
        if corrupt == "kind":
            raw[bad_index, 0:4] = np.frombuffer(np.uint32(99).tobytes(), np.uint8)
        else:
            raw[bad_index, 0:4] = np.frombuffer(np.uint32(xk.TASK_AXPBY).tobytes(), np.uint8)
            rng = np.array([0, 0, 10, 3], np.int64)          # x, y null; lo 10 > hi 3
            raw[bad_index, 8:40] = rng.view(np.uint8)
        dev = torch.from_numpy(bad.view(np.uint8).copy()).cuda()
        executed = ctypes.c_uint64(123)
        rc = xk.lib().xkb_sched_run_noalloc(dev.data_ptr(), ctypes.byref(graph), 1, 1.0, stream, ctypes.byref(executed))
        assert rc == xk.XKB_EINVAL
        assert f"task {bad_index}:".encode() in xk.lib().xkb_last_error()
        assert executed.value == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(b.cpu().numpy(), g)          # no tile was written
    good = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    executed = ctypes.c_uint64()
    xk.check(xk.lib().xkb_sched_run_noalloc(good.data_ptr(), ctypes.byref(graph), 1, 1.0, stream, ctypes.byref(executed)))
    assert executed.value == len(d)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.cpu().numpy(), O.heat_run(g, nx, ny, 2, 0.2))


@pytest.mark.parametrize("limit", [float("inf"), float("nan"), 0.0, -1.0, 3601.0])
def test_noalloc_rejects_unusable_time_limits(limit):
    graph = xk.TaskGraph(0, 0, 0, 0, 0)
    rc = xk.lib().xkb_sched_run_noalloc(None, ctypes.byref(graph), 2, limit, None, None)
    assert rc == xk.XKB_EINVAL
    assert b"time limit" in xk.lib().xkb_last_error()
