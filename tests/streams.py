"""Seeded access-stream generators and the stream file codec used by the tests.

A stream is the list of accesses tasks declare, in spawn order; each record mirrors the
arguments of the reference's access_t constructors (matrix: storage address, ld, offset_m,
offset_n, m, n, sizeof; segment: [a, b)). The 64-byte record layout is the one the oracle
programs read (oracle/access_stream.h) and the one the C-ABI resolver takes
(include/xkrt_b200.h, xkb_access_rec_t).
"""
import numpy as np

MAGIC = 0x314D525453424B58
HANDLE, SEGMENT, MATRIX = 0, 1, 2
R, W, RW, V, D = 1, 2, 3, 4, 8

REC = np.dtype([("task", "<u4"), ("type", "u1"), ("mode", "u1"), ("reserved", "<u2"),
                ("addr", "<u8"), ("ld", "<u8"), ("offset_m", "<u8"), ("offset_n", "<u8"),
                ("m", "<u8"), ("n", "<u8"), ("sizeof_type", "<u8")])
assert REC.itemsize == 64


def write_stream(path, recs):
    with open(path, "wb") as f:
        np.array([MAGIC, len(recs)], dtype="<u8").tofile(f)
        recs.astype(REC).tofile(f)


def read_edges(path):
    e = np.fromfile(path, dtype="<u4")
    return e.reshape(-1, 2)


def from_tuples(tasks):
    """tasks: list of lists of access tuples
    ('m', mode, addr, ld, off_m, off_n, m, n, s), ('s', mode, a, b) or ('h', mode, handle)."""
    rows = []
    for t, accs in enumerate(tasks):
        for a in accs:
            if a[0] == "m":
                _, mode, addr, ld, om, on, m, n, s = a
                rows.append((t, MATRIX, mode, 0, addr, ld, om, on, m, n, s))
            elif a[0] == "h":
                _, mode, h = a
                rows.append((t, HANDLE, mode, 0, h, 0, 0, 0, 0, 0, 0))
            else:
                _, mode, lo, hi = a
                rows.append((t, SEGMENT, mode, 0, lo, hi, 0, 0, 0, 0, 0))
    return np.array(rows, dtype=REC)


def heat_stream(nx, ny, tsx, tsy, steps, base_src=1 << 20, base_dst=None, s=8):
    """The heat-diffusion-2d access pattern (examples/heat-diffusion-2d/src/main.cc:508-581):
    tiles tile_x outer / tile_y inner; access 0 = R on the halo-expanded source tile clipped
    to the grid, access 1 = W on the destination tile clipped to the interior [1, N-1)."""
    if base_dst is None:
        base_dst = base_src + nx * ny * s + 4096
    ntx, nty = -(-nx // tsx), -(-ny // tsy)
    rows = []
    t = 0
    src, dst = base_src, base_dst
    for _ in range(steps):
        for tx in range(ntx):
            for ty in range(nty):
                x, y = tx * tsx, ty * tsy
                x0, y0 = max(x - 1, 0), max(y - 1, 0)
                x1, y1 = min(x + tsx + 1, nx), min(y + tsy + 1, ny)
                rows.append((t, MATRIX, R, 0, src, nx, x0, y0, x1 - x0, y1 - y0, s))
                x0, y0 = max(x, 1), max(y, 1)
                x1, y1 = min(x + tsx, nx - 1), min(y + tsy, ny - 1)
                rows.append((t, MATRIX, W, 0, dst, nx, x0, y0, x1 - x0, y1 - y0, s))
                t += 1
        src, dst = dst, src
    return np.array(rows, dtype=REC)


def microbench_stream(ntasks, seed, n=8192, ld=8192, s=8, align=64, max_side_units=32,
                      base=1 << 30):
    """Dependency microbench shape: 1-4 accesses per task on an n x n matrix (LD=ld),
    rectangles aligned to `align` elements with sides align*U{1..max_side_units},
    modes R 60% / W 20% / RW 20%."""
    rng = np.random.default_rng(seed)
    units = n // align
    rows = []
    for t in range(ntasks):
        na = int(rng.integers(1, 5))
        for _ in range(na):
            mu = int(rng.integers(1, max_side_units + 1)); nu = int(rng.integers(1, max_side_units + 1))
            mu, nu = min(mu, units), min(nu, units)
            xu = int(rng.integers(0, units - mu + 1)); yu = int(rng.integers(0, units - nu + 1))
            r = int(rng.integers(0, 10))
            mode = R if r < 6 else (W if r < 8 else RW)
            rows.append((t, MATRIX, mode, 0, base, ld, xu * align, yu * align, mu * align, nu * align, s))
    return np.array(rows, dtype=REC)


def mixed_stream(ntasks, seed, base=1 << 20, span=1 << 14):
    """Small adversarial mix: matrices of two (ld, sizeof) domains with column wrap-around,
    segments crossing columns, modes R/W/RW/VR/VW/R|D, 1-4 accesses per task."""
    rng = np.random.default_rng(seed)
    modes = [R, W, RW, R | V, W | V, R | D, R, R]
    rows = []
    for t in range(ntasks):
        for _ in range(int(rng.integers(1, 5))):
            mode = modes[int(rng.integers(0, len(modes)))]
            kind = int(rng.integers(0, 3))
            if kind == 2:
                a = base + int(rng.integers(0, span))
                b = a + int(rng.integers(1, span // 4))
                rows.append((t, SEGMENT, mode, 0, a, b, 0, 0, 0, 0, 0))
            else:
                ld, s = (64, 8) if kind == 0 else (48, 4)
                m = int(rng.integers(1, ld + 1)); n = int(rng.integers(1, 9))
                om = int(rng.integers(0, ld)); on = int(rng.integers(0, 24))
                rows.append((t, MATRIX, mode, 0, base, ld, om, on, m, n, s))
    return np.array(rows, dtype=REC)


def handle_concurrent_stream(seed, n=80):
    """Handle accesses of every concurrency -- sequential, commutative, concurrent writes (record
    field `reserved` >> 8 = 1, 2, 4) -- over three handles, one access per handle in a task,
    mixed with segment accesses; the reference's handle map inserts its extra writer tasks
    (include/xkrt/memory/access/handle/dependency-map.hpp:93-137), numbered in creation order just
    before the task that needed them."""
    rng = np.random.default_rng(seed)
    modes = [R, W, RW, R | V, W | V]
    handles = [0x1000, 0x1008, 0x2000]
    rows = []
    for t in range(n):
        order = rng.permutation(len(handles))[: int(rng.integers(1, 3))]
        for h in order:
            mode = modes[int(rng.integers(0, len(modes)))]
            conc = [1, 2, 4, 4][int(rng.integers(0, 4))] if mode & W else [1, 2][int(rng.integers(0, 2))]
            rows.append((t, HANDLE, mode, conc << 8, handles[h], 0, 0, 0, 0, 0, 0))
        if rng.random() < 0.3:
            a = 0x1000 + int(rng.integers(0, 64))
            rows.append((t, SEGMENT, modes[int(rng.integers(0, 3))], 0, a, a + int(rng.integers(1, 64)), 0, 0, 0, 0, 0))
    return np.array(rows, dtype=REC)
