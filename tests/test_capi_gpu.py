"""The XKRT C API over libxkb200, exercised by C programs compiled against include/xkrt_capi.h
(gcc) and linked to the library: the reference's ordering tests, and the heat example --
fused (device tasks only) and mixed with host export tasks -- checked against the oracle."""
import json
import os
import subprocess

import numpy as np
import pytest

import kernels_oracle as O

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(name, tmp_path):
    exe = str(tmp_path / name)
    lib = os.path.join(REPO, "xkaapi_b200")
    subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-Wall", "-Werror", "-D_POSIX_C_SOURCE=200809L", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "capi", name + ".c"), "-o", exe, "-L", lib, "-lxkb200", "-lpthread",
                    "-Wl,-rpath," + lib], check=True)
    return exe


def test_devices_detach_unified_program(torch_cuda, tmp_path):
    """Device and driver objects, the current task, a task completed from another thread after its
    body returned (its successor waits), unified memory used in place (no copies), refused calls."""
    r = subprocess.run([build("api_capi", tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout.strip().splitlines()[-1])["ok"] == 1


def test_driver_interface_program(torch_cuda, tmp_path):
    """Drivers, devices, driver memory and queued transfers, a module image (cubin built here)
    whose kernel runs from a queue and from a CUDA task body (xkrt_task_kernel_launch), device
    memory, file I/O tasks ordered before a reader task, teams, the energy counter."""
    cubin = str(tmp_path / "scale.cubin")
    subprocess.run(["nvcc", "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-o", cubin,
                    os.path.join(REPO, "tests", "capi", "scale_kernel.cu")], check=True)
    r = subprocess.run([build("driver_capi", tmp_path), cubin, str(tmp_path / "scratch.bin")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["ok"] == 1 and "B200" in out["info"]


@pytest.mark.parametrize("threads", [None, 1])
def test_dataflow_host_team(torch_cuda, tmp_path, threads):
    """A non-fused batch runs as a dataflow graph on a team of host threads: independent tasks run
    at the same time, chains keep their order, a detached task completed by another task's body
    releases its successor -- also with a single host thread (a detached task holds none)."""
    env = dict(os.environ)
    if threads:
        env["XKB_HOST_THREADS"] = str(threads)
    r = subprocess.run([build("dataflow_capi", tmp_path)], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    if threads == 1:
        assert out["peak"] == 1
    elif (os.cpu_count() or 1) >= 4:
        assert out["peak"] >= 4 and out["wide_s"] < 48 * 0.020 / 2


def test_streaming_stops_midway(torch_cuda, tmp_path):
    """Short axpby chunks stream window by window; a pass of chunks that must be split stops the
    streaming; the rest runs at the wait behind the streamed windows (with the split) -- y is the
    host's result bit for bit."""
    import re
    env = dict(os.environ, XKB_RESOLVE_CHUNK="16", XKB_TRACE_WAIT="1")
    r = subprocess.run([build("stream_rest_capi", tmp_path)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["mismatches"] == 0 and out["fused"] == 1
    m = re.search(r"(\d+) of (\d+) tasks streamed", r.stderr)
    assert m and 0 < int(m.group(1)) < int(m.group(2)) == out["tasks"]


def test_ordering_programs(torch_cuda, tmp_path):
    r = subprocess.run([build("order_capi", tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    assert out["tasks"] == 6 and out["edges"] >= 4
    assert out["handle_edges"] == 2                    # T6 -> T7 -> T8 on the handle


def test_concurrent_handle_program(torch_cuda, tmp_path):
    """Concurrent writes of a handle: they run after the last sequential write and before the
    next reads, the handle map's two extra writer tasks run (13 tasks), the 18 edges are the
    reference's (two diagrams of dependency-map.hpp), and a concurrent segment access is refused."""
    r = subprocess.run([build("concurrent_capi", tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out == {"x": 482, "ran": 13, "edges": 18, "order": 1, "refused": 1}


@pytest.mark.parametrize("every,chunk", [(0, None), (3, None), (0, 64), (3, 64)])
def test_heat_example(torch_cuda, tmp_path, every, chunk):
    nx, ny, ts, steps = 200, 136, 64, 7
    g = O.heat_init(nx, ny, seed=4)
    g.tofile(tmp_path / "init.bin")
    exe = build("heat_capi", tmp_path)
    env = dict(os.environ)
    if chunk:
        env["XKB_RESOLVE_CHUNK"] = str(chunk)         # resolution in the background while spawning
    r = subprocess.run([exe, str(nx), str(ny), str(ts), str(steps), str(every), str(tmp_path / "init.bin"),
                        str(tmp_path / "out.bin"), str(tmp_path / "sums.txt")], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    stats = json.loads(r.stdout)
    out = np.fromfile(tmp_path / "out.bin").reshape(ny, nx)
    np.testing.assert_array_equal(out, O.heat_run(g, nx, ny, steps, 0.2))
    assert stats["fused"] == (1 if every == 0 else 0)
    assert stats["h2d"] > 0 and stats["d2h"] > 0
    if every:
        for line in open(tmp_path / "sums.txt"):
            s, v = line.split()
            # the export body sums in memory order, one add at a time: cumsum does the same
            assert float(v) == np.cumsum(O.heat_run(g, nx, ny, int(s), 0.2).ravel())[-1]


@pytest.mark.parametrize("chunk,nx,ny,ts,steps,every,waits", [(None, 260, 190, 64, 11, 3, 4), (100, 260, 190, 64, 11, 3, 4),
                                                              (None, 1030, 1030, 16, 16, -1, 5)])
def test_heat_many_waits_one_runtime(torch_cuda, tmp_path, chunk, nx, ny, ts, steps, every, waits):
    """Several xkrt_task_wait in one runtime on registered user memory, each batch resolved anew
    (in the background when the resolver batch is small); the grid equals the oracle's. With
    growing batches (every < 0) the last one needs more page-locked descriptor memory than the
    ones before."""
    g = O.heat_init(nx, ny, seed=23)
    g.tofile(tmp_path / "init.bin")
    env = dict(os.environ)
    if chunk:
        env["XKB_RESOLVE_CHUNK"] = str(chunk)
    r = subprocess.run([build("heat_waits_capi", tmp_path), str(nx), str(ny), str(ts), str(steps), str(every),
                        str(tmp_path / "init.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout)["waits"] == waits
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.bin").reshape(ny, nx), O.heat_run(g, nx, ny, steps, 0.2))


@pytest.mark.parametrize("planner", ["resident", "reference"])
def test_reset_forgets_device_copies(torch_cuda, tmp_path, planner):
    """xkrt_reset between waits (the reference's runtime_t::reset, src/memory/invalidate.cc:66-133):
    the program halves the source grid in host memory after each wait, then resets; every batch
    reads the halved grid, so the result is the oracle's with the same halvings (the device's
    copies of the grid, coherent before the host write, are forgotten)."""
    nx, ny, ts, steps, every = 260, 190, 64, 9, 3
    g = O.heat_init(nx, ny, seed=31)
    g.tofile(tmp_path / "init.bin")
    env = dict(os.environ)
    if planner == "reference":
        env["XKB_PLANNER"] = "reference"
    r = subprocess.run([build("heat_waits_capi", tmp_path), str(nx), str(ny), str(ts), str(steps), str(every),
                        str(tmp_path / "init.bin"), str(tmp_path / "out.bin"), "reset"], capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout)["waits"] == 3
    want = g
    for k in range(steps // every):
        want = O.heat_run(want, nx, ny, every, 0.2)
        if k + 1 < steps // every:
            want = want * 0.5
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.bin").reshape(ny, nx), want)


@pytest.mark.parametrize("protect", ["1", "0"])
def test_reference_mode_registration_splits(torch_cuda, tmp_path, protect):
    """Reference mode on user memory registered with xkrt_memory_register (the grids come from
    malloc, so they are not page-aligned): with the reference's default registration-overflow
    protection the copies the C API executes (XKB_PLAN_RECORD) are the planner's plan for the
    same stream after the two registrations -- the planner's splits are pinned to the reference's
    memory tree by tests/test_planner.py -- and they differ from the plan without them;
    XKAAPI_MEMORY_REGISTER_PROTECT_OVERFLOW=0 gives the plan without them. The grid is the
    oracle's either way."""
    import streams as S
    import xkaapi_b200 as xk
    nx, ny, ts, steps = 200, 136, 64, 5
    g = O.heat_init(nx, ny, seed=41)
    g.tofile(tmp_path / "init.bin")
    env = dict(os.environ, XKB_PLANNER="reference", XKB_PLAN_RECORD=str(tmp_path / "plan.bin"),
               XKAAPI_MEMORY_REGISTER_PROTECT_OVERFLOW=protect)
    r = subprocess.run([build("heat_waits_capi", tmp_path), str(nx), str(ny), str(ts), str(steps), str(steps),
                        str(tmp_path / "init.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.bin").reshape(ny, nx), O.heat_run(g, nx, ny, steps, 0.2))
    recs = S.heat_stream(nx, ny, ts, ts, steps, base_src=out["grid_a"], base_dst=out["grid_b"])

    def plan(registered):
        P = xk.Planner()
        xk.check(xk.lib().xkb_planner_set_writeback_coherent(P._h, 1))   # what the reference mode sets
        if registered:
            P.register(out["grid_a"], nx * ny * 8)
            P.register(out["grid_b"], nx * ny * 8)
        first = 0
        for i in range(len(recs)):
            if i == 0 or recs[i]["task"] != recs[i - 1]["task"]:
                first = i
            P.fetch(recs[i], i - first, 1)
        for i in range(len(recs)):                  # the wait's write-back: every written access, spawn order
            if recs[i]["mode"] & S.W:
                P.fetch(recs[i], 1, 0)
        return P.copies()

    key = lambda q: q[np.lexsort(tuple(q[:, k] for k in range(13, -1, -1)))]
    done = key(np.fromfile(tmp_path / "plan.bin", dtype=np.int64).reshape(-1, 14))
    with_reg, without = key(plan(True)), key(plan(False))
    assert len(with_reg) != len(without)
    np.testing.assert_array_equal(done, with_reg if protect == "1" else without)


def test_spawn_generic_detachable_count_and_ocr(torch_cuda, tmp_path):
    """xkrt_task_spawn_generic: a detachable task spawned with an initial counter of 2 completes
    only after two xkrt_task_detachable_decr from another thread (its successor sees both), one
    with counter 0 completes when its body returns, and device tasks spawned with a non-default
    ocr_access run and compute the right y (one GPU owns every access)."""
    r = subprocess.run([build("spawn_generic_capi", tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    assert json.loads(r.stdout.strip().splitlines()[-1]) == {"order": 1, "early": 1, "axpby": 1}


def test_partly_locked_registration_and_range_checks(torch_cuda, tmp_path):
    """A registration made while tasks are pending, touching locked memory, stays unlocked except
    the page it shares with the locked piece; axpby tasks on a vector starting in that page run
    and are exact (copies are cut at the locked piece's end). An axpby whose element range leaves
    its vector's region is refused with XKB_EINVAL instead of running past the region's mirror."""
    r = subprocess.run([build("register_pieces_capi", tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    assert json.loads(r.stdout.strip().splitlines()[-1]) == {"ok": 1, "refused": 1}
