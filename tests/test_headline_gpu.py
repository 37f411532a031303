"""The headline heat configuration end to end, at full size, through the drop-in C API.

examples/heat_xkrt spawns the 16384 x 16384 heat graph of 128 x 128 tile tasks for 500 steps
(8,192,000 tasks) through xkrt_task_spawn_with_format_with_accesses and calls xkrt_task_wait,
with the runtime's default settings: resolution in streamed windows of about a million
accesses while the program spawns, the windows run on the persistent scheduler, the written
blocks copied back to the host grids. The grid it writes back is compared with the threaded C
oracle (oracle/heat_oracle.c, the update of examples/heat-diffusion-2d/src/main.cc:408-421) run
for the same 500 steps on the same seeded grid: bit-exact in FP64; in FP32 storage bit-exact
against the oracle's FP32-storage run and within 1e-5 relative of the FP64 result."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import kernels_oracle as O

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(REPO, "xkaapi_b200", "examples", "heat_xkrt")
N, TS, STEPS, C = 16384, 128, 500, 0.2


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _oracle_run(g, dtype):
    """STEPS double-buffered Jacobi steps of the C oracle on all host threads."""
    L = O.c_oracle()
    step = L.xk_oracle_heat_step_f64 if dtype == np.float64 else L.xk_oracle_heat_step_f32
    a = np.array(g, dtype=dtype, copy=True)          # the oracle steps in place: never on the caller's grid
    b = a.copy()
    nt = _threads()
    for _ in range(STEPS):
        step(a.ctypes.data, b.ctypes.data, N, N, N, C, nt)
        a, b = b, a
    return a


@pytest.fixture(scope="module")
def headline(tmp_path_factory):
    d = tmp_path_factory.mktemp("headline")
    g = O.heat_init(N, N, seed=42)
    g.tofile(d / "init.bin")
    return d, g


def _run_example(d, f32):
    out = d / f"out{f32}.bin"
    r = subprocess.run([EXE, str(N), str(N), str(TS), str(STEPS), "1", str(f32), str(d / "init.bin"), str(out)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["tasks"] == (N // TS) ** 2 * STEPS and line["fused"] == 1
    return np.fromfile(out).reshape(N, N), line


def test_headline_f64_bit_exact(torch_cuda, headline):
    d, g = headline
    out, line = _run_example(d, 0)
    ref = _oracle_run(g, np.float64)
    assert line["edges"] > 70_000_000                 # the whole 500-step graph was resolved
    np.testing.assert_array_equal(out, ref)
    np.save(d / "ref64.npy", ref)


def test_headline_f32_storage(torch_cuda, headline):
    d, g = headline
    out, _ = _run_example(d, 1)
    ref32 = _oracle_run(g.astype(np.float32), np.float32)
    np.testing.assert_array_equal(out, ref32.astype(np.float64))
    p = d / "ref64.npy"
    ref64 = np.load(p) if p.exists() else _oracle_run(g, np.float64)
    rel = float(np.max(np.abs(out - ref64)) / np.max(np.abs(ref64)))
    assert rel <= 1e-5, rel
