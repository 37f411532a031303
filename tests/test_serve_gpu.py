"""Served stream: heat graphs of mixed sizes, step counts and precisions arrive over time and
run concurrently under an HBM budget. Each request's result equals the same request served
alone and the oracle (bit-exact: FP64 and FP32 storage)."""
import ctypes

import numpy as np
import pytest

import kernels_oracle as O
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu


def make_requests(specs, tiles=None):
    reqs = (xk.Request * len(specs))()
    bufs = []
    for k, (r, (t, n, steps, f32, seed)) in enumerate(zip(reqs, specs)):
        buf = np.zeros((n, n), dtype=np.float32 if f32 else np.float64)
        bufs.append(buf)
        ts = 64 if tiles is None else tiles[k]
        r.arrival_s, r.nx, r.ny, r.ts, r.steps, r.f32, r.seed, r.c = t, n, n, ts, steps, f32, seed, 0.2
        r.result = buf.ctypes.data
    return reqs, bufs


def test_mixed_stream_equals_alone_and_oracle(torch_cuda):
    rng = np.random.default_rng(3)
    specs = []
    t = 0.0
    for k in range(24):
        t += float(rng.exponential(0.004))
        n = int(rng.choice([64, 96, 128, 200, 256, 384]))
        specs.append((t, n, int(rng.integers(1, 13)), int(k % 2), 1000 + k))
    # budget for only a few grids at once: admission has to wait for memory to be freed
    srv = xk.Server(budget_bytes=6 << 20, slots=4, ctas_per_graph=64, max_seconds=60.0)
    reqs, bufs = make_requests(specs)
    srv.run(reqs)
    for r in reqs:
        assert r.finish_s >= r.start_s >= r.arrival_s - 1e-9
    alone = xk.Server(budget_bytes=6 << 20, slots=1, max_seconds=60.0)
    for i, (spec, buf) in enumerate(zip(specs, bufs)):
        solo, sbuf = make_requests([(0.0,) + spec[1:]])
        alone.run(solo)
        np.testing.assert_array_equal(buf, sbuf[0])
        t, n, steps, f32, seed = spec
        dt = np.float32 if f32 else np.float64
        ref = O.heat_run(O.serve_init(n, n, seed, dt), n, n, steps, 0.2, dtype=dt)
        np.testing.assert_array_equal(buf, ref)
    srv.close(); alone.close()


def test_request_over_budget_is_rejected(torch_cuda):
    srv = xk.Server(budget_bytes=1 << 20, slots=2)
    reqs, _ = make_requests([(0.0, 1024, 2, 0, 1)])          # 2 x 8 MiB grids > 1 MiB budget
    with pytest.raises(xk.XkbError) as e:
        srv.run(reqs)
    assert e.value.code == xk.XKB_ERANGE
    srv.close()


def test_device_loop_with_inputs_equals_launch_mode(torch_cuda, monkeypatch):
    """The device-resident loop (one persistent kernel for every request) with initial grids
    given as host inputs, against the per-request launch mode (XKB_SERVE_MODE=launch) on the
    same trace, and the oracle: every result bit for bit, with 16 slots so many requests share
    the kernel at once, step counts odd and even, one request of zero steps."""
    rng = np.random.default_rng(11)
    specs, t = [], 0.0
    for k in range(40):
        t += float(rng.exponential(0.002))
        n = int(rng.choice([96, 130, 256, 320, 512]))
        specs.append((t, n, 0 if k == 7 else int(rng.integers(1, 16)), int(k % 3 == 0), 500 + k))
    results = {}
    for mode in ("device", "launch"):
        if mode == "launch":
            monkeypatch.setenv("XKB_SERVE_MODE", "launch")
        reqs, bufs = make_requests(specs)
        inputs = []
        for r, (_, n, _, f32, seed) in zip(reqs, specs):
            g = np.ascontiguousarray(O.serve_init(n, n, seed, np.float32 if f32 else np.float64))
            inputs.append(g)
            r.input = g.ctypes.data
        srv = xk.Server(budget_bytes=64 << 20, slots=16, max_seconds=60.0)
        srv.run(reqs)
        srv.close()
        results[mode] = bufs
        for r in reqs:
            assert r.finish_s >= r.start_s >= r.arrival_s - 1e-9
    for (t, n, steps, f32, seed), a, b in zip(specs, results["device"], results["launch"]):
        dt = np.float32 if f32 else np.float64
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, O.heat_run(O.serve_init(n, n, seed, dt), n, n, steps, 0.2, dtype=dt))


def test_tile_sides_of_a_stream_equal_the_oracle(torch_cuda):
    """Requests of one stream tiled 64^2, 128^2 and 256^2 (a strip sweeps several 128-row pieces of
    a 256^2 tile; ragged last tiles), FP64 and FP32 storage, in the device-resident loop: every
    result equals the oracle bit for bit."""
    specs, tiles = [], []
    for k, (n, ts) in enumerate([(300, 256), (520, 256), (400, 128), (258, 64), (640, 256), (384, 128)]):
        specs.append((0.001 * k, n, 3 + k, k % 2, 2000 + k))
        tiles.append(ts)
    srv = xk.Server(budget_bytes=64 << 20, slots=4, max_seconds=60.0)
    reqs, bufs = make_requests(specs, tiles)
    srv.run(reqs)
    srv.close()
    for (t, n, steps, f32, seed), buf in zip(specs, bufs):
        dt = np.float32 if f32 else np.float64
        np.testing.assert_array_equal(buf, O.heat_run(O.serve_init(n, n, seed, dt), n, n, steps, 0.2, dtype=dt))
