"""The dependency oracle restatement against golden edge sets produced by the reference's own
dependency trees (tests/golden/make_golden.py), plus oracle self-checks. CPU only."""
import os
import subprocess

import numpy as np
import pytest

import streams as S

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = np.load(os.path.join(REPO, "tests", "golden", "deps_golden.npz"))
CASES = sorted(k[:-len("__stream")] for k in GOLDEN.files if k.endswith("__stream"))


def run_oracle(recs, tmp_path):
    p = str(tmp_path / "s.bin")
    S.write_stream(p, recs)
    subprocess.run([os.path.join(REPO, "oracle", "_bin", "deps_oracle"), p, str(tmp_path / "o")],
                   check=True, capture_output=True)
    return S.read_edges(str(tmp_path / "o.edges"))


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_golden(case, tmp_path):
    edges = run_oracle(GOLDEN[case + "__stream"], tmp_path)
    np.testing.assert_array_equal(edges, GOLDEN[case + "__edges"])


def test_known_answer_orderings():
    # reference tests/task-dependency-interval.cc and tests/task-dependency-interval-matrix.cc:
    # both build the chain T0 -> T1 -> T2
    for case in ("ref_interval_chain", "ref_interval_matrix_chain"):
        e = set(map(tuple, GOLDEN[case + "__edges"].tolist()))
        assert {(0, 1), (1, 2)} <= e, (case, e)


def test_heat_oracle_properties():
    import kernels_oracle as O
    g = O.heat_init(40, 30, seed=1)
    assert (g[0] == 0).all() and (g[:, 0] == 0).all() and (g[-1] == 0).all() and (g[:, 39] == 0).all()
    out = O.heat_run(g, 40, 30, 5, 0.2)
    assert (out[0] == 0).all() and (out[:, 39] == 0).all()          # Dirichlet boundary preserved
    # tile decomposition == whole step (the task graph computes the same grid)
    ref = O.heat_step(g, g.copy(), 40, 30, 0.2)
    t = g.copy()
    for tx in range(3):
        for ty in range(3):
            O.heat_tile(g, t, 40, 30, tx, ty, 16, 11, 0.2)
    np.testing.assert_array_equal(t, ref)


def test_c_oracle_equals_numpy_oracle():
    import kernels_oracle as O
    L = O.c_oracle()
    for dt, fn in ((np.float64, L.xk_oracle_heat_step_f64), (np.float32, L.xk_oracle_heat_step_f32)):
        g = O.heat_init(97, 61, 100, seed=2).astype(dt)
        ref = O.heat_step(g, g.copy(), 97, 61, 0.2)
        out = g.copy()
        fn(g.ctypes.data, out.ctypes.data, 97, 61, 100, 0.2, 4)
        np.testing.assert_array_equal(out, ref)
    x = np.linspace(-1, 1, 1001); y = np.linspace(3, -2, 1001); ref = O.axpby(0.3, x, -1.7, y)
    L.xk_oracle_axpby(1001, 0.3, x.ctypes.data, -1.7, y.ctypes.data, 2)
    np.testing.assert_array_equal(y, ref)


def test_reference_runtime_heat_equals_oracle(tmp_path):
    """The reference's own host-only runtime (oracle/_ref/ref_heat, built from its sources)
    running the heat example's task graph produces the oracle's grid bit for bit."""
    import kernels_oracle as O
    exe = os.path.join(REPO, "oracle", "_ref", "ref_heat")
    if not os.path.exists(exe):
        pytest.skip("reference runtime not built (oracle/ref/build_ref.sh)")
    nx, ny, ts, steps = 300, 200, 64, 9
    g = O.heat_init(nx, ny, seed=3)
    g.tofile(tmp_path / "init.bin")
    env = dict(os.environ, DRIVERS="host,4", XKRT_DRIVERS="host,4")
    subprocess.run([exe, str(nx), str(ny), str(ts), str(steps), str(tmp_path / "init.bin"), str(tmp_path / "out.bin")],
                   env=env, check=True, capture_output=True, cwd=str(tmp_path), timeout=120)
    out = np.fromfile(tmp_path / "out.bin").reshape(ny, nx)
    np.testing.assert_array_equal(out, O.heat_run(g, nx, ny, steps, 0.2))


AXPBY_GOLDEN = np.load(os.path.join(REPO, "tests", "golden", "axpby_golden.npz"))
AXPBY_CASES = sorted(k[:-len("__params")] for k in AXPBY_GOLDEN.files if k.endswith("__params"))


@pytest.mark.parametrize("case", AXPBY_CASES)
def test_axpby_chain_oracle_matches_reference_runtime(case):
    """The oracle's restatement of the seeded axpby task chains (generator + y = a*x + b*y per
    chunk, in spawn order) equals the final y of the reference's own host runtime bit for bit."""
    import kernels_oracle as O
    n, passes, seed, cmin, cmax = (int(v) for v in AXPBY_GOLDEN[case + "__params"])
    x, y, chunks = O.axpby_chain(n, passes, seed, cmin, cmax)
    assert len(chunks) == int(AXPBY_GOLDEN[case + "__tasks"][0])
    np.testing.assert_array_equal(O.axpby_chain_run(x, y, chunks), AXPBY_GOLDEN[case + "__y"])


WRAP = np.load(os.path.join(REPO, "tests", "golden", "wrap_golden.npz"))
WRAP_CASES = sorted(k[:-len("__stream")] for k in WRAP.files if k.endswith("__stream"))


def _closure(edges, n):
    reach = [set() for _ in range(n)]
    succ = [[] for _ in range(n)]
    for p, s in edges:
        succ[p].append(s)
    for t in range(n - 1, -1, -1):
        for s in succ[t]:
            reach[t].add(s)
            reach[t] |= reach[s]
    return reach


@pytest.mark.parametrize("case", WRAP_CASES)
def test_wrapped_tiles_pinned_divergence(case, tmp_path):
    """Tiles that wrap the leading dimension: the reference's tree is not point-wise there
    (include/xkrt/memory/access/blas/dependency-tree.hpp:228-256 applies a PUT to whole split-off
    nodes that meet the access's other rect), the restatement and the GPU resolver are. The
    fixture holds both edge sets; the restatement reproduces its point-wise set exactly, so the
    difference to the reference is exactly the recorded one -- and every edge only the point-wise
    set has is one the reference orders too, through other tasks."""
    recs = WRAP[case + "__stream"]
    mine = run_oracle(recs, tmp_path)
    np.testing.assert_array_equal(mine, WRAP[case + "__pointwise_edges"])
    ref = set(map(tuple, WRAP[case + "__ref_edges"].tolist()))
    ours = set(map(tuple, mine.tolist()))
    n = int(recs["task"].max()) + 1
    reach = _closure(ref, n)
    assert all(s in reach[p] for p, s in ours - ref)
    assert any(int(r["offset_m"]) + int(r["m"]) > int(r["ld"]) for r in recs if r["type"] == S.MATRIX)
