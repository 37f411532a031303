"""GPU parity of the heat-diffusion tile body against the numpy oracle (bit-exact in FP64;
FP32-storage within 1e-5 relative of the FP64 oracle)."""
import numpy as np
import pytest

import kernels_oracle as O
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu
C = 0.2


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("nx,ny,ld", [(64, 64, 64), (130, 97, 130), (131, 77, 136), (3, 3, 3), (5, 200, 7),
                                      (1024, 1024, 1024), (257, 129, 257)])
def test_step_f64_bit_exact(torch_cuda, nx, ny, ld):
    torch = torch_cuda
    g = O.heat_init(nx, ny, ld, seed=nx * 1000 + ny)
    ref = O.heat_step(g, g.copy(), nx, ny, C)
    s, d = to_dev(torch, g), to_dev(torch, g)
    xk.heat_step(s, d, nx, ny, ld, C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), ref)


@pytest.mark.parametrize("nx,ny,tsx,tsy", [(64, 64, 16, 16), (1024, 1024, 128, 128), (200, 136, 64, 48),
                                           (130, 130, 128, 128), (97, 61, 33, 17)])
def test_tiles_f64_bit_exact(torch_cuda, nx, ny, tsx, tsy):
    torch = torch_cuda
    g = O.heat_init(nx, ny, seed=3)
    ref = g.copy()
    s, d = to_dev(torch, g), to_dev(torch, g)
    ntx, nty = -(-nx // tsx), -(-ny // tsy)
    for tx in range(ntx):
        for ty in range(nty):
            O.heat_tile(g, ref, nx, ny, tx, ty, tsx, tsy, C)
            xk.heat_tile(s, d, nx, ny, nx, tx, ty, tsx, tsy, C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), ref)
    # a tile beyond the grid writes nothing
    xk.heat_tile(s, d, nx, ny, nx, ntx + 1, 0, tsx, tsy, C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), ref)


def test_run_100_steps_f64_1024(torch_cuda):
    """Config: 1024x1024 FP64, c=0.2, Dirichlet 0, 100 double-buffered steps."""
    torch = torch_cuda
    nx = ny = 1024
    g = O.heat_init(nx, ny, seed=42)
    ref = O.heat_run(g, nx, ny, 100, C)
    a, b = to_dev(torch, g), to_dev(torch, g)
    for _ in range(100):
        xk.heat_step(a, b, nx, ny, nx, C)
        a, b = b, a
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.cpu().numpy(), ref)


@pytest.mark.parametrize("nx,ny", [(512, 384), (131, 77)])
def test_f32_storage_matches_oracle_and_fp64(torch_cuda, nx, ny):
    torch = torch_cuda
    g64 = O.heat_init(nx, ny, seed=5)
    g32 = g64.astype(np.float32)
    steps = 20
    ref32 = O.heat_run(g32, nx, ny, steps, C, dtype=np.float32)
    ref64 = O.heat_run(g64, nx, ny, steps, C)
    a, b = to_dev(torch, g32), to_dev(torch, g32)
    for _ in range(steps):
        xk.heat_step(a, b, nx, ny, nx, C)
        a, b = b, a
    torch.cuda.synchronize()
    out = a.cpu().numpy()
    np.testing.assert_array_equal(out, ref32)          # same rounding as the FP32-storage oracle
    rel = np.abs(out.astype(np.float64) - ref64).max() / np.abs(ref64).max()
    assert rel <= 1e-5, rel                            # FP32-storage error bound vs FP64


def test_f32_tiles_bit_exact(torch_cuda):
    torch = torch_cuda
    nx, ny, ts = 300, 260, 128
    g = O.heat_init(nx, ny, seed=9).astype(np.float32)
    ref = g.copy()
    s, d = to_dev(torch, g), to_dev(torch, g)
    for tx in range(-(-nx // ts)):
        for ty in range(-(-ny // ts)):
            O.heat_tile(g, ref, nx, ny, tx, ty, ts, ts, C)
            xk.heat_tile(s, d, nx, ny, nx, tx, ty, ts, ts, C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), ref)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("tsy", [1, 2, 3, 5, 6, 7, 12, 13, 17, 36, 128])
def test_tile_column_blocks_bit_exact(torch_cuda, dtype, tsy):
    """Tile strips sweep their columns in blocks (FP64: 2 columns, FP32: 6) -- whole blocks with
    no per-column checks, then one checked block for the rest: tile widths that are multiples of
    a block, one column past one, and shorter than one, FP64 and FP32 storage."""
    torch = torch_cuda
    nx, ny, tsx = 200, 149, 64
    g = O.heat_init(nx, ny, seed=tsy)
    if dtype == "f32":
        g = g.astype(np.float32)
    ref = g.copy()
    s, d = to_dev(torch, g), to_dev(torch, g)
    for tx in range(-(-nx // tsx)):
        for ty in range(-(-ny // tsy)):
            O.heat_tile(g, ref, nx, ny, tx, ty, tsx, tsy, C)
            xk.heat_tile(s, d, nx, ny, nx, tx, ty, tsx, tsy, C)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), ref)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_heat_norms_fp64_checks(torch_cuda, dtype):
    """xkb_heat_norms: boundary max, L2 norm and the step's residual in FP64, against numpy on
    the same grids; the residual is 0 for FP64 storage and the float rounding for FP32."""
    torch = torch_cuda
    nx, ny = 300, 170
    g = O.heat_init(nx, ny, seed=31)
    npdt = np.float64 if dtype == "f64" else np.float32
    src = torch.from_numpy(g.astype(npdt)).cuda()
    dst = src.clone()
    xk.heat_step(src, dst, nx, ny, nx, 0.2)
    n = xk.heat_norms(src, dst, nx, ny, nx, 0.2)
    d = dst.cpu().numpy().astype(np.float64)
    exact = O.heat_step(g.astype(npdt).astype(np.float64), g.astype(np.float64).copy(), nx, ny, 0.2)
    interior = d[1:-1, 1:-1]
    assert n["boundary_max_abs"] == 0.0
    assert abs(n["l2_norm"] - np.sqrt((interior ** 2).sum())) <= 1e-12 * n["l2_norm"]
    assert n["interior_max_abs"] == np.abs(interior).max()
    res = np.abs(interior - exact[1:-1, 1:-1]).max()
    assert n["residual_max_abs"] == res
    if dtype == "f64":
        assert res == 0.0
    else:
        assert 0 < res <= 2.0 ** -24 * n["interior_max_abs"]
