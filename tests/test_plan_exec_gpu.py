"""Reference-layout execution on the GPU: every heat tile task runs on its own per-access
replicas, made coherent by executing the planner's copies (H2D, batched D2D), with the
replica-layout tile body. The grid assembled from the last step's written replicas must equal
the oracle bit-exactly -- the plan moves exactly the data the tile bodies need.

(The reference's write-back path copies from the block's view on its LARGEST allocation without
checking that view is coherent (fetch_list_to_host_setup_partition,
include/xkrt/memory/access/blas/memory-tree.hpp:1135-1145); for heat that is a stale halo
replica. The planner reproduces that plan exactly -- see tests/test_planner.py -- so the result
is read from the written replicas here instead.)"""
import numpy as np
import pytest

import kernels_oracle as O
import streams as S
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny,ts,steps", [(256, 256, 64, 5), (200, 136, 64, 4)])
def test_heat_through_plan(torch_cuda, nx, ny, ts, steps):
    torch = torch_cuda
    c = 0.2
    g = O.heat_init(nx, ny, seed=11)
    A = torch.from_numpy(g.copy()).pin_memory(); B = torch.from_numpy(g.copy()).pin_memory()
    recs = S.heat_stream(nx, ny, ts, ts, steps, base_src=A.data_ptr(), base_dst=B.data_ptr())
    P = xk.Planner()
    views, tasks = [], []
    first = 0
    for i in range(len(recs)):
        if i == 0 or recs[i]["task"] != recs[i - 1]["task"]:
            first = i
        views.append(P.fetch(recs[i], i - first, 1))
        tasks.append(P.copies(take=True))          # the copies this access needs, in plan order
    sizes = P.allocations()
    bufs = [torch.empty(int(sz), dtype=torch.uint8, device="cuda") for sz in sizes]
    ptrs = [b.data_ptr() for b in bufs]
    ntx, nty = -(-nx // ts), -(-ny // ts)
    per = ntx * nty
    for t in range(int(recs["task"].max()) + 1):
        idx = np.nonzero(recs["task"] == t)[0]
        for i in idx:
            if len(tasks[i]):
                xk.plan_execute(tasks[i], ptrs)
        k = t % per
        tx, ty = k // nty, k % nty
        vs, vd = views[idx[0]], views[idx[1]]
        src = int(ptrs[vs[0]] + vs[1]); dst = int(ptrs[vd[0]] + vd[1])
        ld_s, ld_d = int(vs[2]), int(vd[2])
        # launcher re-basing (examples/heat-diffusion-2d/src/main.cc:214-219)
        if tx == 0: dst -= 8
        else: src += 8
        if ty == 0: dst -= 8 * ld_d
        else: src += 8 * ld_s
        xk.check(xk.lib().xkb_diffusion_views(xk.F64, torch.cuda.current_stream().cuda_stream, src, ld_s, dst, ld_d,
                                              tx, ty, ts, ts, nx, ny, c))
    torch.cuda.synchronize()
    # assemble the final grid from the last step's written replicas (W access = index 1)
    out = np.zeros((ny, nx))
    host_bufs = [b.cpu().numpy() for b in bufs]
    for t in range(per * (steps - 1), per * steps):
        i = np.nonzero(recs["task"] == t)[0][1]
        r, v = recs[i], views[i]
        m, n, ld = int(r["m"]), int(r["n"]), int(v[2])
        raw = host_bufs[v[0]][v[1]:v[1] + 8 * (ld * (n - 1) + m)].view(np.float64)
        tile = np.lib.stride_tricks.as_strided(raw, shape=(n, m), strides=(8 * ld, 8))
        out[int(r["offset_n"]):int(r["offset_n"]) + n, int(r["offset_m"]):int(r["offset_m"]) + m] = tile
    np.testing.assert_array_equal(out, O.heat_run(g, nx, ny, steps, c))


def test_whole_plan_in_one_call(torch_cuda):
    """The full copy list of a multi-access stream in one xkb_plan_execute call (batches per
    access) moves the same bytes as executing access by access."""
    torch = torch_cuda
    host = torch.arange(256 * 256, dtype=torch.float64).reshape(256, 256).pin_memory()   # the whole 256 x 256 matrix
    recs = S.microbench_stream(7, 3, n=256, ld=256, align=16, max_side_units=6, base=host.data_ptr())
    recs["mode"] = S.R                              # reads only: every copy is H2D or D2D
    P = xk.Planner(); P.plan(recs, 1)
    copies = P.copies(); sizes = P.allocations()
    a = [torch.zeros(int(s), dtype=torch.uint8, device="cuda") for s in sizes]
    b = [torch.zeros(int(s), dtype=torch.uint8, device="cuda") for s in sizes]
    xk.plan_execute(copies, [t.data_ptr() for t in a])
    for k in np.unique(copies[:, 0] * 16 + copies[:, 1]):
        xk.plan_execute(copies[copies[:, 0] * 16 + copies[:, 1] == k], [t.data_ptr() for t in b])
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
