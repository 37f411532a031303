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


def test_noalloc_run_matches_allocating_scheduler_twice(torch_cuda):
    torch = torch_cuda
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
