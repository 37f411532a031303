"""Autotuner for the heat-diffusion task graph on the persistent scheduler.

Searches the tile shape (square tiles, 128-1024 cells per side) and the number of warps that
execute one task (1, 2, 4 or 8 -- i.e. tasks in flight per CTA = 8 / warps) by running a short
graph of each candidate on the device and timing the persistent kernel with CUDA events.
Objective: HBM bytes moved per second (16 B per cell per step in FP64, 8 B in FP32 storage),
which is what the tile shape trades off (small tiles: more scheduling work per byte; large
tiles: fewer tasks to balance over the SMs)."""
import time

from . import Resolver, Scheduler, heat_access_records, heat_task_descs


def autotune_heat(a, b, nx, ny, ld=None, tiles=(128, 256, 512, 1024), teams=(1, 2, 4, 8), steps=6,
                  c=0.2, f32=False, stream=None, reps=2):
    """a, b: the two grids (torch CUDA tensors). Returns (best, results) where best is a dict
    {tile, team, ms_per_step, GBps} and results lists every candidate."""
    import torch
    ld = nx if ld is None else ld
    esz = 4 if f32 else 8
    results = []
    for ts in tiles:
        if ts > max(nx, ny):
            continue
        res = Resolver(stream)
        res.add(heat_access_records(nx, ny, ts, ts, 0, steps, a.data_ptr(), b.data_ptr(), esize=esz, ld=ld))
        g = res.graph()
        sch = Scheduler(stream)
        sch.set_tasks(heat_task_descs((a.data_ptr(), b.data_ptr()), nx, ny, ld, ts, ts, steps, c, f32=f32))
        for team in teams:
            sch.set_team(team)
            ctx = torch.cuda.stream(stream) if stream is not None else torch.cuda.stream(torch.cuda.current_stream())
            with ctx:
                sch.run(g); sch.wait()
                best_ms = None
                for _ in range(reps):
                    sch.run(g); sch.wait()
                    ms = sch.kernel_ms()
                    best_ms = ms if best_ms is None else min(best_ms, ms)
            per_step = best_ms / steps
            gbs = 2.0 * esz * (nx - 2) * (ny - 2) / (per_step / 1e3) / 1e9
            results.append({"tile": ts, "team": team, "ms_per_step": round(per_step, 4), "GBps": round(gbs, 1),
                            "tasks_per_s": round(g.ntasks / (best_ms / 1e3))})
        sch.close(); res.close()
    best = max(results, key=lambda r: r["GBps"])
    return best, results
