"""ORACLE -- test infrastructure only (imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker; never by the product).

CPU restatement of the task bodies on the path, in numpy (each operation a separate IEEE
double operation, so no fused multiply-add can occur):

* heat_step: the heat-diffusion-2d update of examples/heat-diffusion-2d/src/main.cc:408-421
  (update_cpu) with DX = DY = 1 and c = ALPHA*DT/(DX*DY):
      D(i,j) = S(i,j) + c*( ((S(i+1,j) - 2S(i,j)) + S(i-1,j)) + ((S(i,j+1) - 2S(i,j)) + S(i,j-1)) )
  on interior cells only; boundary cells of dst are left untouched. Grids are column-major
  with leading dimension ld: numpy arrays of shape (ny, ld), cell (i, j) at G[j, i]
  (GRID(G,I,J,L) = G[J*L+I], examples/heat-diffusion-2d/include/heat/consts.h:90).
  FP32-storage mode: cells read as float32, promoted to double, updated in double, rounded
  once to float32.
* heat_tile: the same update restricted to one tile task's cells
  (examples/heat-diffusion-2d/src/main.cc:508-566 decomposition, src/kernels/diffusion.cu:107-128).
* axpby: y = (a*x) + (b*y) (no reference kernel exists; examples/task-axpby.cc:43-52 is the
  byte-wise analogue).
* heat_init: the seeded synthetic grid: interior U[0,1) from numpy's PCG64 generator with the
  given seed, boundary 0 (Dirichlet).
"""
import numpy as np


def heat_init(nx, ny, ld=None, seed=42, dtype=np.float64):
    ld = nx if ld is None else ld
    g = np.zeros((ny, ld), dtype=np.float64)
    rng = np.random.default_rng(seed)
    g[1:ny - 1, 1:nx - 1] = rng.random((ny - 2, nx - 2))
    return g.astype(dtype)


def _update(S, c):
    """Interior update of a (ny, nx') view S (float64). Returns the (ny-2, nx'-2) block."""
    s = S[1:-1, 1:-1]
    a = (S[1:-1, 2:] - 2.0 * s) + S[1:-1, :-2]      # rows i+1, i-1 (contiguous dim)
    b = (S[2:, 1:-1] - 2.0 * s) + S[:-2, 1:-1]      # cols j+1, j-1
    return s + c * (a + b)


def heat_tile(src, dst, nx, ny, tile_x, tile_y, tsx, tsy, c):
    """Update the interior cells of tile (tile_x, tile_y) of dst from src (in place on dst)."""
    x0, y0 = tile_x * tsx, tile_y * tsy
    rx0, rx1 = max(x0, 1), min(x0 + tsx, nx - 1)
    cy0, cy1 = max(y0, 1), min(y0 + tsy, ny - 1)
    if rx0 >= rx1 or cy0 >= cy1:
        return dst
    S = src[cy0 - 1:cy1 + 1, rx0 - 1:rx1 + 1].astype(np.float64)
    dst[cy0:cy1, rx0:rx1] = _update(S, c).astype(dst.dtype)
    return dst


def heat_step(src, dst, nx, ny, c):
    if nx >= 3 and ny >= 3:
        S = src[:ny, :nx].astype(np.float64)
        dst[1:ny - 1, 1:nx - 1] = _update(S, c).astype(dst.dtype)
    return dst


def heat_run(grid, nx, ny, steps, c, dtype=np.float64):
    """Double-buffered Jacobi: returns the grid after `steps` steps."""
    a = grid.astype(dtype).copy()
    b = a.copy()
    for _ in range(steps):
        heat_step(a, b, nx, ny, c)
        a, b = b, a
    return a


def axpby(a, x, b, y):
    return (a * x) + (b * y)


def c_oracle():
    """ctypes handle on oracle/_bin/libheat_oracle.so (C restatement, POSIX threads)."""
    import ctypes
    import os
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_bin", "libheat_oracle.so")
    L = ctypes.CDLL(p)
    i64, vp, dbl, ci = ctypes.c_int64, ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    for name in ("xk_oracle_heat_step_f64", "xk_oracle_heat_step_f32"):
        getattr(L, name).argtypes = [vp, vp, i64, i64, i64, dbl, ci]
    L.xk_oracle_axpby.argtypes = [i64, dbl, vp, dbl, vp, ci]
    return L


def serve_init(nx, ny, seed, dtype=np.float64):
    """Initial grid of a served request: interior cell k = j*nx + i gets U[0,1) from a splitmix64
    hash of (seed * 0x100000001b3 + k), taking the top 53 bits; boundary 0."""
    k = np.arange(nx * ny, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) * np.uint64(0x100000001B3) + k
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    v = (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    g = v.reshape(ny, nx)
    g[0, :] = 0; g[-1, :] = 0; g[:, 0] = 0; g[:, -1] = 0
    return g.astype(dtype)


_GAMMA = 0x9E3779B97F4A7C15
_M64 = (1 << 64) - 1


def _mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def axpby_chain(n, passes, seed, cmin, cmax):
    """The seeded axpby task-chain workload (the draw sequence of the reference-runtime driver
    oracle/ref/ref_axpby.cc and the example xkaapi_b200/examples/axpby_xkrt.c): a splitmix64
    stream s += gamma; x[i], then y[i] = 2u - 1 (u = top 53 bits / 2^53); per pass a, b = 4u - 2,
    then chunk lengths floor(exp(log cmin + (log cmax - log cmin) u) / 8) elements (at least 1),
    the first one of a pass shortened to 1 + floor(u * len). Returns (x, y, chunks) with chunks a
    list of (lo, hi, a, b) in spawn order."""
    import math
    k = np.arange(1, 2 * n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * np.uint64(_GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    x, y = 2.0 * u[:n] - 1.0, 2.0 * u[n:] - 1.0
    s = (seed + 2 * n * _GAMMA) & _M64

    def unit():
        nonlocal s
        s = (s + _GAMMA) & _M64
        return (_mix64(s) >> 11) * (1.0 / 9007199254740992.0)

    lmin, lmax = math.log(cmin), math.log(cmax)
    chunks = []
    for _ in range(passes):
        a = 4.0 * unit() - 2.0
        b = 4.0 * unit() - 2.0
        at, first = 0, True
        while at < n:
            ln = max(int(math.exp(lmin + (lmax - lmin) * unit()) / 8.0), 1)
            if first:
                ln, first = 1 + int(unit() * ln), False
            hi = min(at + ln, n)
            chunks.append((at, hi, a, b))
            at = hi
    return x, y, chunks


def axpby_chain_run(x, y, chunks):
    """y after every chunk task in spawn order (each element once per pass)."""
    y = y.copy()
    for lo, hi, a, b in chunks:
        y[lo:hi] = axpby(a, x[lo:hi], b, y[lo:hi])
    return y
