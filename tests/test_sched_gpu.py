"""Resolved task graphs executed by the device scheduler in its three forms (persistent
kernel, one launch per task, CUDA graph): results bit-exact against the oracle."""
import numpy as np
import pytest

import kernels_oracle as O
import streams as S
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu
C = 0.2


class _DevView:
    def __init__(self, ptr, n, typestr="<i4"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def heat_graph(torch, nx, ny, ts, steps, f32=False, seed=42):
    dt = np.float32 if f32 else np.float64
    g = O.heat_init(nx, ny, seed=seed).astype(dt)
    a = torch.from_numpy(g).cuda(); b = torch.from_numpy(g).cuda()
    esz = 4 if f32 else 8
    recs = S.heat_stream(nx, ny, ts, ts, steps, base_src=a.data_ptr(), base_dst=b.data_ptr(), s=esz)
    res = xk.Resolver()
    res.add(recs)
    descs = xk.heat_task_descs((a.data_ptr(), b.data_ptr()), nx, ny, nx, ts, ts, steps, C, f32=f32)
    return g, a, b, res, descs


@pytest.mark.parametrize("form", [xk.FORM_PERSISTENT, xk.FORM_PLAIN, xk.FORM_GRAPH])
@pytest.mark.parametrize("nx,ny,ts,steps", [(1024, 1024, 128, 100), (300, 200, 64, 7)])
def test_heat_forms_bit_exact(torch_cuda, form, nx, ny, ts, steps):
    torch = torch_cuda
    if form == xk.FORM_GRAPH and steps > 20:
        steps = 20                           # keep graph instantiation short
    g, a, b, res, descs = heat_graph(torch, nx, ny, ts, steps)
    sch = xk.Scheduler()
    sch.set_tasks(descs)
    sch.run(res.graph(), form)
    n = sch.wait()
    if form == xk.FORM_PERSISTENT:
        assert n == len(descs)
    out = (a if steps % 2 == 0 else b).cpu().numpy()
    np.testing.assert_array_equal(out, O.heat_run(g, nx, ny, steps, C))
    sch.close(); res.close()


def test_heat_f32_persistent(torch_cuda):
    torch = torch_cuda
    nx = ny = 512
    g, a, b, res, descs = heat_graph(torch, nx, ny, 128, 30, f32=True)
    sch = xk.Scheduler(); sch.set_tasks(descs); sch.run(res.graph()); sch.wait()
    out = a.cpu().numpy()
    np.testing.assert_array_equal(out, O.heat_run(g, nx, ny, 30, C, dtype=np.float32))
    ref64 = O.heat_run(g.astype(np.float64), nx, ny, 30, C)
    assert np.abs(out.astype(np.float64) - ref64).max() / np.abs(ref64).max() <= 1e-5


def test_persistent_small_grid_many_ctas(torch_cuda):
    # more CTAs than ready tasks at any time: idle CTAs wait on queue slots and still finish
    torch = torch_cuda
    g, a, b, res, descs = heat_graph(torch, 256, 256, 64, 40)
    sch = xk.Scheduler(); sch.set_grid(600); sch.set_tasks(descs); sch.run(res.graph()); sch.wait()
    np.testing.assert_array_equal(a.cpu().numpy(), O.heat_run(g, 256, 256, 40, C))


def axpby_chain(torch, n, passes, seed):
    """y = a*x + b*y over seeded chunkings whose boundaries move between passes (segment
    accesses: R on the x chunk, RW on the y chunk)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n); y = rng.uniform(-1, 1, n)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    tasks, chunks = [], []
    for p in range(passes):
        a, b = rng.uniform(-2, 2, 2)
        off = int(rng.integers(1, 97))
        cuts = [0, off]
        while cuts[-1] < n:
            cuts.append(min(n, cuts[-1] + int(rng.integers(1, max(2, n // 6)))))
        for lo, hi in zip(cuts[:-1], cuts[1:]):
            if lo < hi:
                tasks.append([("s", S.R, dx.data_ptr() + 8 * lo, dx.data_ptr() + 8 * hi),
                              ("s", S.RW, dy.data_ptr() + 8 * lo, dy.data_ptr() + 8 * hi)])
                chunks.append((lo, hi, a, b))
    ref = y.copy()
    for lo, hi, a, b in chunks:
        ref[lo:hi] = O.axpby(a, x[lo:hi], b, ref[lo:hi])
    descs = np.zeros(len(chunks), dtype=xk.axpby_desc_dtype())
    descs["kind"] = xk.TASK_AXPBY; descs["x"] = dx.data_ptr(); descs["y"] = dy.data_ptr()
    descs["lo"] = [c[0] for c in chunks]; descs["hi"] = [c[1] for c in chunks]
    descs["a"] = [c[2] for c in chunks]; descs["b"] = [c[3] for c in chunks]
    return S.from_tuples(tasks), descs, dy, ref


@pytest.mark.parametrize("form", [xk.FORM_PERSISTENT, xk.FORM_PLAIN, xk.FORM_GRAPH])
def test_axpby_chains(torch_cuda, form):
    torch = torch_cuda
    recs, descs, dy, ref = axpby_chain(torch, 200_003, 10, 7)
    res = xk.Resolver(); res.add(recs)
    sch = xk.Scheduler(); sch.set_tasks(descs); sch.run(res.graph(), form); sch.wait()
    np.testing.assert_array_equal(dy.cpu().numpy(), ref)


def test_timeout_returns_error_and_context_survives(torch_cuda):
    """A task whose wait counter never reaches zero: the persistent CTAs give up after the
    time limit, the kernel returns, xkb_sched_wait reports XKB_ETIMEDOUT; the context is
    then reused for a valid graph."""
    torch = torch_cuda
    ptr = torch.zeros(3, dtype=torch.int32, device="cuda")          # no edges
    succ = torch.zeros(1, dtype=torch.int32, device="cuda")
    npred = torch.tensor([0, 1], dtype=torch.int32, device="cuda")   # task 1 waits for nobody's release
    g = xk.TaskGraph(2, 0, ptr.data_ptr(), succ.data_ptr(), npred.data_ptr())
    descs = np.zeros(2, dtype=xk.task_desc_dtype())                 # two no-op tasks
    sch = xk.Scheduler(); sch.set_tasks(descs); sch.set_timeout(0.2); sch.set_grid(4)
    sch.run(g)
    with pytest.raises(xk.XkbError) as e:
        sch.wait()
    assert e.value.code == xk.XKB_ETIMEDOUT
    g2, a, b, res, d2 = heat_graph(torch, 128, 128, 64, 4)
    sch.set_tasks(d2); sch.run(res.graph()); sch.wait()
    np.testing.assert_array_equal(a.cpu().numpy(), O.heat_run(g2, 128, 128, 4, C))


@pytest.mark.parametrize("team", [1, 2, 4, 8])
def test_heat_persistent_team_sizes(torch_cuda, team):
    torch = torch_cuda
    g, a, b, res, descs = heat_graph(torch, 300, 200, 64, 9)
    sch = xk.Scheduler(); sch.set_team(team); sch.set_tasks(descs); sch.run(res.graph())
    assert sch.wait() == len(descs)
    np.testing.assert_array_equal(b.cpu().numpy(), O.heat_run(g, 300, 200, 9, C))


@pytest.mark.parametrize("team", [1, 8])
def test_axpby_chains_team_sizes(torch_cuda, team):
    torch = torch_cuda
    recs, descs, dy, ref = axpby_chain(torch, 50_001, 6, 3)
    res = xk.Resolver(); res.add(recs)
    sch = xk.Scheduler(); sch.set_team(team); sch.set_tasks(descs); sch.run(res.graph()); sch.wait()
    np.testing.assert_array_equal(dy.cpu().numpy(), ref)


@pytest.mark.parametrize("steps", [1, 2, 7, 10])
def test_periodic_heat_one_launch(torch_cuda, steps):
    """Three resolved two-step windows -> periodic form; one persistent launch runs all steps
    (a half window at the end for odd step counts) and gives the oracle's grid."""
    torch = torch_cuda
    nx, ny, ts = 300, 200, 64
    g0 = O.heat_init(nx, ny, seed=21)
    a = torch.from_numpy(g0).cuda(); b = torch.from_numpy(g0).cuda()
    res = xk.Resolver()
    res.add(xk.heat_access_records(nx, ny, ts, ts, 0, 6, a.data_ptr(), b.data_ptr()))
    per_step = (-(-nx // ts)) * (-(-ny // ts))
    pg = res.periodic(2 * per_step)
    sch = xk.Scheduler()
    sch.set_tasks(xk.heat_task_descs((a.data_ptr(), b.data_ptr()), nx, ny, nx, ts, ts, 2, C))
    sch.run_periodic(pg, (steps + 1) // 2, per_step if steps % 2 else 2 * per_step)
    assert sch.wait() == steps * per_step
    out = (a if steps % 2 == 0 else b).cpu().numpy()
    np.testing.assert_array_equal(out, O.heat_run(g0, nx, ny, steps, C))


def test_periodic_rejects_aperiodic_graph(torch_cuda):
    recs = S.microbench_stream(30, 1, n=512, ld=512)
    res = xk.Resolver(); res.add(recs)
    with pytest.raises(xk.XkbError):
        res.periodic(10)


@pytest.mark.parametrize("nx,ny,ts,steps,f32,team", [
    (1024, 768, 128, 12, False, 2), (300, 200, 64, 9, False, 1), (300, 200, 100, 9, False, 8),
    (301, 203, 64, 6, False, 2),                       # rows not 16-byte aligned: register body
    (516, 260, 128, 10, True, 2), (514, 130, 64, 6, True, 4), (1000, 1000, 96, 8, True, 1)])
def test_bulk_staged_body_matches_register_body(torch_cuda, nx, ny, ts, steps, f32, team):
    """The bulk-staged tile body (default) and the register body give the oracle's grid bit for
    bit, for FP64 and FP32 storage, tiles that are not a multiple of the strip, and grids whose
    rows cannot be staged (odd FP64 / non-multiple-of-4 FP32 widths fall back)."""
    torch = torch_cuda
    dt = np.float32 if f32 else np.float64
    want = O.heat_run(O.heat_init(nx, ny, seed=5), nx, ny, steps, C, dtype=dt)
    for bulk in (True, False):
        g, a, b, res, descs = heat_graph(torch, nx, ny, ts, steps, f32=f32, seed=5)
        sch = xk.Scheduler(); sch.set_team(team); sch.set_staging(bulk); sch.set_tasks(descs)
        sch.run(res.graph())
        assert sch.wait() == len(descs)
        np.testing.assert_array_equal((a if steps % 2 == 0 else b).cpu().numpy(), want)
        sch.close(); res.close()
