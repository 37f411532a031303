"""Host side of the heat-diffusion-2d task graph: the tile tasks the reference example spawns
(examples/heat-diffusion-2d/src/main.cc:508-581), as access records for the resolver and as
task descriptors for the device scheduler. Vectorised with numpy so graphs of millions of
tile tasks are generated in seconds."""
import numpy as np

from . import TASK_HEAT_F32, TASK_HEAT_F64, task_desc_dtype

ACCESS_REC = np.dtype([("task", "<u4"), ("type", "u1"), ("mode", "u1"), ("reserved", "<u2"),
                       ("addr", "<u8"), ("ld", "<u8"), ("offset_m", "<u8"), ("offset_n", "<u8"),
                       ("m", "<u8"), ("n", "<u8"), ("sizeof_type", "<u8")])
MATRIX, R, W = 2, 1, 2


def _tiles(nx, ny, tsx, tsy):
    ntx, nty = -(-nx // tsx), -(-ny // tsy)
    tx = np.repeat(np.arange(ntx, dtype=np.int64), nty)       # tile_x outer, tile_y inner
    ty = np.tile(np.arange(nty, dtype=np.int64), ntx)
    return tx, ty


def heat_access_records(nx, ny, tsx, tsy, step0, nsteps, grid_a, grid_b, esize=8, ld=None):
    """Access records of steps [step0, step0+nsteps): per tile task, access 0 = R on the
    halo-expanded source tile clipped to the grid, access 1 = W on the destination tile clipped
    to the interior [1, N-1) (main.cc:544-561). Even steps read grid_a, odd steps grid_b."""
    ld = nx if ld is None else ld
    tx, ty = _tiles(nx, ny, tsx, tsy)
    per = len(tx)
    x, y = tx * tsx, ty * tsy
    r_x0, r_y0 = np.maximum(x - 1, 0), np.maximum(y - 1, 0)
    r_x1, r_y1 = np.minimum(x + tsx + 1, nx), np.minimum(y + tsy + 1, ny)
    w_x0, w_y0 = np.maximum(x, 1), np.maximum(y, 1)
    w_x1, w_y1 = np.minimum(x + tsx, nx - 1), np.minimum(y + tsy, ny - 1)
    recs = np.zeros(2 * per * nsteps, dtype=ACCESS_REC)
    for k in range(nsteps):
        s = step0 + k
        src, dst = (grid_a, grid_b) if s % 2 == 0 else (grid_b, grid_a)
        blk = recs[2 * per * k:2 * per * (k + 1)]
        t = np.arange(per, dtype=np.uint32) + np.uint32(per * s)
        rd, wr = blk[0::2], blk[1::2]
        for v, mode, base, x0, y0, x1, y1 in ((rd, R, src, r_x0, r_y0, r_x1, r_y1),
                                              (wr, W, dst, w_x0, w_y0, w_x1, w_y1)):
            v["task"] = t; v["type"] = MATRIX; v["mode"] = mode; v["addr"] = base; v["ld"] = ld
            v["offset_m"] = x0; v["offset_n"] = y0; v["m"] = x1 - x0; v["n"] = y1 - y0; v["sizeof_type"] = esize
    return recs


def heat_task_descs(grids, nx, ny, ld, tsx, tsy, steps, c, f32=False):
    """Task descriptors of the same tile tasks, in spawn order. grids = (A, B) device pointers."""
    tx, ty = _tiles(nx, ny, tsx, tsy)
    per = len(tx)
    d = np.zeros(per * steps, dtype=task_desc_dtype())
    for s in range(steps):
        blk = d[s * per:(s + 1) * per]
        blk["kind"] = TASK_HEAT_F32 if f32 else TASK_HEAT_F64
        blk["src"], blk["dst"] = (grids[0], grids[1]) if s % 2 == 0 else (grids[1], grids[0])
        blk["ld"], blk["nx"], blk["ny"], blk["c"] = ld, nx, ny, c
        blk["x0"] = tx * tsx; blk["x1"] = np.minimum(tx * tsx + tsx, nx)
        blk["y0"] = ty * tsy; blk["y1"] = np.minimum(ty * tsy + tsy, ny)
    return d
