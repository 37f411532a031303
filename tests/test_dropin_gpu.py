"""Drop-in check: the reference's own test programs and its heat-diffusion-2d example, compiled
UNMODIFIED from the reference tree against this repository's include/ tree and linked against
libxkb200.so (tests/dropin/build_dropin.sh, run by the build where the reference tree is
present), run on the GPU.

* tests/task-dependency.cc, task-format-host.cc: a task built by hand (thread_t::allocate_task,
  task_t / task_dep_info_t placement, access_t constructor, thread_t::resolve,
  runtime_t::task_commit) runs its host body before runtime_t::deinit returns.
* tests/task-dependency-interval.cc, -interval-matrix.cc, -handle.cc: three tasks whose segment,
  matrix or handle accesses conflict must run in spawn order; each body asserts its argument is
  the number of bodies run before it. Their bodies are declared `void func(task_t *)` while the
  reference's runtime calls host bodies as f(runtime, device, task) (src/task.cc:336), so on the
  reference itself these asserts read the runtime object instead of the task and fail. This
  library calls bodies the same way by default; XKB_CXX_HOST_BODY=task passes the task first
  instead, which is what these older programs expect, and makes their order checks meaningful.
* tests/init.cc, deinit.cc, sync.cc, task-format.cc: runtime start and end, a wait with nothing
  spawned, an empty task format.
* tests/task-gpu-empty.cc: a hand-built DEVICE task (RW matrix access on malloc'd memory) whose
  format has only a host function. The reference runs the host function when the device's target
  has none (src/task.cc:322-330); here such a task runs as a host task on the host team.
* tests/memory-register-async-legacy.cc: memory_register_async of an unaligned malloc'd range,
  then a wait.
* tests/memory-register-assisted.cc, -assisted-unregister.cc: three overlapping registrations of
  one buffer (the reference registers only the new pages each time), the whole buffer distributed
  to the GPU by distribute_async over its union, then overlapping unregistrations (one twice).
  Here overlapping registrations merge into one region.
* tests/api/c/task-with-access.c: a C team task with a segment access (api/c/include/xkrt/xkrt.h).
* examples/heat-diffusion-2d: the whole example (32 x 32 FP32 grid, 1000 steps, placement through
  distribute_async, a CUDA-target tile body launched by task_detachable_kernel_launch on the
  queue's stream, ten host export tasks reading the grid back for VTK files); its last frame is
  compared with the example's update formula evaluated in FP32 with numpy (the file holds two
  decimals per cell).
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "tests", "dropin", "_bin")


def _exe(name):
    p = os.path.join(BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (tests/dropin/build_dropin.sh needs the reference tree at build time)")
    return p


def _run(name, tmp_path, env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    r = subprocess.run([_exe(name)], cwd=tmp_path, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, f"{name} exited {r.returncode}: {r.stderr[-1500:]}"
    return r


@pytest.mark.parametrize("name", ["task-dependency", "task-format-host", "init", "deinit", "sync", "task-format",
                                  "task-gpu-empty", "memory-register-async-legacy", "memory-register-assisted",
                                  "memory-register-assisted-unregister"])
def test_reference_task_programs(torch_cuda, tmp_path, name):
    _run(name, tmp_path)


@pytest.mark.parametrize("name", ["task-dependency-interval", "task-dependency-interval-matrix", "task-dependency-handle"])
def test_reference_ordering_programs(torch_cuda, tmp_path, name):
    _run(name, tmp_path, {"XKB_CXX_HOST_BODY": "task"})


def test_reference_c_team_task(torch_cuda, tmp_path):
    r = _run("task-with-access", tmp_path)
    assert r.stdout.splitlines().count("in") == 1


def _heat_reference_frame(steps):
    """The example's update (examples/heat-diffusion-2d/src/kernels/diffusion.cu:107-128 with
    include/heat/consts.h: TYPE float, NX = NY = 32, boundary 100, interior 0) in float32."""
    nx = 32
    alpha = np.float32(1.11e-4)
    dx = np.float32(1.0)
    dt = np.float32(0.5) * (dx * dx * dx * dx) / (np.float32(2.0) * alpha * (dx * dx + dx * dx))
    c = alpha * dt / (dx * dx)
    g = np.zeros((nx, nx), np.float32)
    g[0, :] = g[-1, :] = g[:, 0] = g[:, -1] = np.float32(100)
    for _ in range(steps):
        s = g
        d = s.copy()
        d[1:-1, 1:-1] = s[1:-1, 1:-1] + c * ((s[1:-1, 2:] - np.float32(2) * s[1:-1, 1:-1] + s[1:-1, :-2]) / (dx * dx) +
                                             (s[2:, 1:-1] - np.float32(2) * s[1:-1, 1:-1] + s[:-2, 1:-1]) / (dx * dx))
        g = d
    return g


def test_reference_heat_example(torch_cuda, tmp_path):
    _run("heat-diffusion-2d", tmp_path)
    frames = sorted(f for f in os.listdir(tmp_path) if f.startswith("temperature_grid_") and f.endswith(".vtk"))
    assert len(frames) == 10
    with open(os.path.join(tmp_path, frames[-1])) as fh:
        lines = fh.read().splitlines()
    k = lines.index("LOOKUP_TABLE default")
    vals = np.array([float(v) for v in lines[k + 1:k + 1 + 32 * 32]], np.float64).reshape(32, 32)
    ref = _heat_reference_frame(1000).astype(np.float64)        # frame 9 = the grid after step 999
    assert np.max(np.abs(vals - ref)) <= 0.0101
    assert vals[16, 16] > 1.0                                    # heat reached the centre
