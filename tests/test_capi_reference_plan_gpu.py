"""The coherency plan the C API executes, in reference mode (XKB_PLANNER=reference), against the
reference's own memory tree.

In reference mode the runtime makes each task's accesses coherent with the reference's decisions
(KBLASMemoryTree::fetch, include/xkrt/memory/access/blas/memory-tree.hpp:1738-1874: one device
allocation per access unless an older one already has a view on every block, H2D from the host
for blocks never on the device, D2D between views of the GPU, the written view the only coherent
copy), runs the tasks one at a time in spawn order (the canonical schedule the golden plans were
made with), executes every planned copy, and the bodies use the per-access allocations. With
XKB_PLAN_RECORD the runtime appends every copy it executes to a file.

Checked here, for the heat graph of tests/golden/plan_golden.npz (1024^2 FP64, 128^2 tiles,
4 steps; golden made by the reference's memory tree, tests/golden/make_golden.py):
* the H2D and D2D copies the C API executed equal the golden plan record for record (host
  addresses compared relative to each grid);
* the grid read back equals the oracle's, bit for bit -- for the program's own CUDA kernel
  (examples/heat_cxx, C++ source API) and for the library's tile body (examples/heat_xkrt).
"""
import json
import os
import subprocess

import numpy as np
import pytest

import kernels_oracle as O

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(REPO, "tests", "golden", "plan_golden.npz"))
CASE = "plan_heat_1024_t128_s4"
N, TS, STEPS = 1024, 128, 4


def _run(exe, args, tmp_path, record):
    env = dict(os.environ, XKB_PLANNER="reference", XKB_PLAN_RECORD=str(record), HEAT_CXX_PLACE="0")
    r = subprocess.run([os.path.join(REPO, "xkaapi_b200", "examples", exe)] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.strip().splitlines()]


def _normalise(q, bases_from, bases_to, size):
    """Host addresses (source of H2D, destination of D2H) moved from one pair of grid bases to another."""
    q = q.copy()
    for col, kind in ((5, 0), (9, 1)):
        sel = q[:, 2] == kind
        for b_from, b_to in zip(bases_from, bases_to):
            hit = sel & (q[:, col] >= b_from) & (q[:, col] < b_from + size)
            q[hit, col] += b_to - b_from
    return q


def _sorted(q):
    return q[np.lexsort(tuple(q[:, k] for k in range(13, -1, -1)))] if len(q) else q


def _golden():
    stream = G[CASE + "__stream"]
    bases = sorted(set(int(a) for a in stream["addr"]))
    return G[CASE + "__plan"], bases


@pytest.mark.parametrize("exe", ["heat_cxx", "heat_xkrt"])
def test_capi_reference_plan_and_grid(torch_cuda, tmp_path, exe):
    g = O.heat_init(N, N, seed=4)
    g.tofile(tmp_path / "init.bin")
    record = tmp_path / "plan.bin"
    args = [N, N, TS, STEPS, 1] + ([] if exe == "heat_cxx" else [0]) + [tmp_path / "init.bin", tmp_path / "out.bin"]
    lines = _run(exe, args, tmp_path, record)
    grids = [lines[-1]["grid_a"], lines[-1]["grid_b"]]
    assert lines[-1]["tasks"] == (N // TS) ** 2 * STEPS
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.bin").reshape(N, N), O.heat_run(g, N, N, STEPS, 0.2))

    q = np.fromfile(record, dtype=np.int64).reshape(-1, 14)
    dev = q[q[:, 2] != 1]                         # H2D and D2D of the tasks' fetches
    wb = q[q[:, 2] == 1]                          # the write-back at the wait
    gold, gbases = _golden()
    mine = _sorted(_normalise(dev, grids, gbases, N * N * 8))
    np.testing.assert_array_equal(mine, gold)
    # the write-back: the reference's fetch to the host of every written access moves the interior
    # of both grids back once (the later fetches of a block already on the host copy nothing)
    assert int((wb[:, 11] * wb[:, 12] * wb[:, 13]).sum()) == 2 * (N - 2) * (N - 2) * 8


@pytest.mark.parametrize("exe,budget", [("heat_cxx", "12M"), ("heat_xkrt", "12M"), ("heat_xkrt", "3M")])
def test_capi_device_budget_smaller_than_the_grids(torch_cuda, tmp_path, exe, budget):
    """Reference mode with XKB_DEVICE_BUDGET below the two grids (2 x 8 MiB): the per-access
    allocations share one budget, old ones are evicted (blocks whose only copy they hold written
    back to the host first) and the grid is still the oracle's, bit for bit."""
    n, ts, steps = 1024, 128, 8
    g = O.heat_init(n, n, seed=12)
    g.tofile(tmp_path / "init.bin")
    env = dict(os.environ, XKB_PLANNER="reference", XKB_DEVICE_BUDGET=budget)
    args = [n, n, ts, steps, 1] + ([] if exe == "heat_cxx" else [0]) + [tmp_path / "init.bin", tmp_path / "out.bin"]
    r = subprocess.run([os.path.join(REPO, "xkaapi_b200", "examples", exe)] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    np.testing.assert_array_equal(np.fromfile(tmp_path / "out.bin").reshape(n, n), O.heat_run(g, n, n, steps, 0.2))
