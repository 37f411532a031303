"""Benchmark of the B200 dataflow hot path (one JSON line on rank 0).

Workload (headline): the batched heat-diffusion-2d task graph -- a 16384 x 16384 FP64 grid,
128 x 128 tile tasks (16384 per Jacobi step: R on the halo-expanded source tile, W on the
destination tile), 500 double-buffered steps = 8,192,000 tile tasks -- dependencies resolved by
the GPU resolver, executed by the persistent device scheduler. One bench "step" = one
execution of the whole 500-step graph. Metric: tasks/s (whole job, all ranks).

e2e: the same graph through the drop-in XKRT C API (xkaapi_b200/examples/heat_xkrt): every bench
step spawns the 8,192,000 tasks with their accesses and calls xkrt_task_wait, which resolves the
dependencies on the GPU, copies both grids in from pinned host memory, runs the graph and copies
the written blocks back -- timed spawn -> wait, as the reference's runtime is timed.

Beside it: the same graph's first two steps in the plain one-launch-per-task form and as a CUDA
graph (the fused/plain ratio), the whole-step stencil kernel's HBM GB/s (FP64 and FP32
storage), the resolver on the dependency microbench (65,536 tasks, 1-4 accesses on an 8192^2
FP64 matrix), and the CPU baseline: a bounded sample of the same heat graph on the reference's
own host-only runtime built from its sources (oracle/_ref/ref_heat) with all host threads, or the
C restatement of the tile body on the host's cores where that binary is absent.

--impl reference times the reference's own CPU implementation of the path -- its host-only
runtime built from its sources (oracle/_ref/ref_heat) running the same heat graph on all host
threads -- on bounded samples of the same workload (the C restatement of the tile body if that
binary is absent).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

NX = NY = 16384
TS = 128
STEPS = 500
COEF = 0.2
SEED = 42
HBM_FALLBACK = 6650.0


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the persistent kernel from the committed ncu summary."""
    try:
        with open(os.path.join(HERE, "profiles", "traffic.json")) as f:
            return json.load(f).get("sched_persistent_kernel_bytes_per_launch")
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev, self.proc, self.f = dev, None, None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush(); self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) > 8:
                for k, name in enumerate(names):
                    if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(gpus):
    import torch
    rank = int(os.environ.get("RANK", "0")); world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The largest x over all ranks (every rank calls it in the same order; NCCL reduces a device
    tensor, gloo a host one)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, world, seconds_this_rank):
    """Whole-job throughput of `world` replicas: every rank's units over the slowest rank's time."""
    return world * units_per_rank / max_over_ranks(seconds_this_rank, world)


def cells_all(nx, ny):
    return (nx - 2) * (ny - 2)


def build_heat_graph(xk, torch, a, b, nx, ny, ts, steps, stream, batch_steps=25, esize=8):
    res = xk.Resolver(stream)
    t0 = time.perf_counter()
    for s0 in range(0, steps, batch_steps):
        res.add(xk.heat_access_records(nx, ny, ts, ts, s0, min(batch_steps, steps - s0), a.data_ptr(), b.data_ptr(),
                                       esize=esize))
    g = res.graph()
    torch.cuda.synchronize()
    return res, g, time.perf_counter() - t0


_CPU_GRIDS = {}


def cpu_heat_sample(nthreads, steps=None, n=NX, target_s=10.0):
    """C restatement of the heat tile bodies on the host: Jacobi steps of the n x n FP64 grid.
    steps=None: run one step, then enough more to make about target_s seconds of CPU work."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import kernels_oracle as O
    L = O.c_oracle()
    if n not in _CPU_GRIDS:
        g = O.heat_init(n, n, seed=SEED)
        _CPU_GRIDS[n] = (g, g.copy())
    a, b = _CPU_GRIDS[n]
    done, t_all = 0, 0.0
    plan = steps if steps is not None else 1
    while True:
        t0 = time.perf_counter()
        for _ in range(plan):
            L.xk_oracle_heat_step_f64(a.ctypes.data, b.ctypes.data, n, n, n, COEF, nthreads)
            a, b = b, a
        t_all += time.perf_counter() - t0
        done += plan
        if steps is not None or t_all >= target_s * 0.8:
            break
        plan = max(1, min(50, int(target_s / (t_all / done)) - done))
    _CPU_GRIDS[n] = (a, b)
    tasks = done * (-(-n // TS)) ** 2
    return tasks / t_all, t_all, tasks


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


REF_HEAT = os.path.join(HERE, "oracle", "_ref", "ref_heat")


REF_FAILURES = []          # runs of the reference binaries that ended abnormally (kept for the line)


def _ref_run(cmd, env, timeout=600, tries=3):
    """Run a reference harness; an abnormal end (the reference's host runtime now and then dies
    of a signal in the middle of a run, before its result line) is recorded and the run is made
    again, up to `tries` times. A result line printed before a crash is kept."""
    for _ in range(tries):
        with tempfile.TemporaryDirectory() as d:
            r = subprocess.run(cmd, env=env, cwd=d, capture_output=True, text=True, timeout=timeout)
        lines = [l for l in r.stdout.strip().splitlines() if l.startswith("{")]
        if r.returncode != 0:
            tail = [l for l in r.stderr.splitlines() if "[LOGGER]" not in l][-3:]
            REF_FAILURES.append({"cmd": os.path.basename(cmd[0]) + " " + " ".join(cmd[1:]), "rc": r.returncode,
                                 "result_kept": bool(lines), "stderr": " | ".join(tail)[-200:]})
        if lines:
            return json.loads(lines[-1])
    raise RuntimeError(f"reference run {os.path.basename(cmd[0])} failed {tries} times: {REF_FAILURES[-1]}")


def ref_heat_sample(nthreads, steps, n=NX, ts=TS):
    """The reference's own host-only runtime (built from its sources by oracle/ref/build_ref.sh)
    running `steps` Jacobi steps of the n x n heat graph with ts^2 tile tasks on `nthreads`
    host threads; returns (tasks/s, seconds, tasks) as the harness times spawn -> task_wait."""
    env = dict(os.environ, DRIVERS=f"host,{nthreads}", XKRT_DRIVERS=f"host,{nthreads}")
    out = _ref_run([REF_HEAT, str(n), str(n), str(ts), str(steps)], env)
    return out["tasks_per_s"], out["seconds"], out["tasks"]


def cpu_baseline_sample(target_s=10.0):
    """CPU baseline on this host: the reference runtime when it was built, else the C
    restatement of the tile body. About target_s seconds of CPU work."""
    cores = host_threads()
    why = None
    if os.path.exists(REF_HEAT):
        try:
            return _ref_baseline(cores, target_s)
        except Exception as ex:              # keep the bench line; say why the port stands in
            why = str(ex)[:300]
    v, secs, tasks = cpu_heat_sample(cores, steps=None, target_s=target_s)
    out = {"value": round(v, 1), "unit": "tasks/s", "cores": cores, "kind": "port",
           "sample": f"{tasks // (NX // TS) ** 2} Jacobi steps of the {NX}^2 FP64 grid ({tasks} tile tasks, {secs:.1f} s), "
                     "C restatement of the tile body on POSIX threads"}
    if why:
        out["reference_failed"] = why
    if REF_FAILURES:
        out["reference_abnormal_ends"] = REF_FAILURES
    return out


def _ref_baseline(cores, target_s):
    v, secs, tasks = ref_heat_sample(cores, 1)
    steps = max(1, min(200, int(target_s / max(secs, 1e-3))))
    v, secs, tasks = ref_heat_sample(cores, steps)
    out = {"value": round(v, 1), "unit": "tasks/s", "cores": cores, "kind": "reference",
           "sample": f"{steps} Jacobi steps of the {NX}^2 FP64 heat graph ({tasks} tile tasks of {TS}^2, {secs:.1f} s): "
                     f"the reference's own host-only runtime (DRIVERS=host,{cores}) with a host-format tile body"}
    if REF_FAILURES:
        out["reference_abnormal_ends"] = REF_FAILURES
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = host_threads()
    use_ref = os.path.exists(REF_HEAT)
    why = None
    sample_steps = 3
    if use_ref:
        try:
            for _ in range(args.warmup):
                ref_heat_sample(cores, 1)
        except Exception as ex:              # the port stands in; the line says why
            use_ref, why = False, str(ex)[:300]
    if not use_ref:
        for _ in range(args.warmup):
            cpu_heat_sample(cores, steps=1)
    tasks, secs = 0, 0.0
    for _ in range(args.steps):
        if use_ref:
            try:
                _, s, n = ref_heat_sample(cores, sample_steps)
            except Exception as ex:          # three abnormal ends in a row: the port times the rest
                use_ref, why = False, str(ex)[:300]
                _, s, n = cpu_heat_sample(cores, steps=None, target_s=5.0)
        else:
            _, s, n = cpu_heat_sample(cores, steps=None, target_s=5.0)
        tasks += n; secs += s
    v = tasks / secs
    kind = "reference" if use_ref else "port"
    sample = (f"{sample_steps} Jacobi steps of the {NX}^2 FP64 heat graph per bench step on the reference's own host-only "
              f"runtime (DRIVERS=host,{cores}), timed spawn -> task_wait" if use_ref else
              "Jacobi steps of the 16384^2 FP64 grid, about 5 s per bench step (C restatement of the tile body)")
    print(json.dumps({
        "impl": "reference", "metric": "tasks/s", "value": round(v, 1), "unit": "tasks/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"batched heat-diffusion-2d: {NX}x{NY} FP64 grid, {TS}x{TS} tile tasks; each bench step "
                               "times a bounded sample of Jacobi steps on the host", "parallelism": f"{cores} host threads"},
        "cpu_baseline": dict({"value": round(v, 1), "unit": "tasks/s", "cores": cores, "kind": kind, "sample": sample},
                             **({"reference_failed": why} if why else {}),
                             **({"reference_abnormal_ends": REF_FAILURES} if REF_FAILURES else {})),
        "e2e": {"value": round(v, 1), "unit": "tasks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


HEAT_XKRT = os.path.join(HERE, "xkaapi_b200", "examples", "heat_xkrt")


def capi_e2e(reps, world, local, warm=1):
    """End to end through the XKRT C API (xkaapi_b200/examples/heat_xkrt, the heat example
    written against include/xkrt_capi.h): per repetition, spawn every tile task of the graph
    with its R/W accesses, then xkrt_task_wait -- GPU dependency resolution, H2D of both grids
    from pinned host memory, the persistent-scheduler run, D2H of the written blocks -- timed
    from the first spawn to the return of the wait, as the reference's runtime is timed on the
    same graph. `warm` untimed repetitions first. Returns the e2e object (whole job over ranks)."""
    env = dict(os.environ)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = vis.split(",")[local] if vis else str(local)
    r = subprocess.run([HEAT_XKRT, str(NX), str(NY), str(TS), str(STEPS), str(warm + reps)], env=env,
                       capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"heat_xkrt failed: {r.stderr[-600:]}")
    lines = [json.loads(l) for l in r.stdout.strip().splitlines()][warm:]
    secs = max_over_ranks(sum(l["seconds"] for l in lines), world)
    tasks = sum(l["tasks"] for l in lines)
    phases = {k: round(statistics.median(l[k] for l in lines), 1)
              for k in ("resolve_ms", "coherency_ms", "run_ms", "writeback_ms")}
    phases["spawn_ms"] = round(statistics.median(l["spawn_s"] for l in lines) * 1e3, 1)
    return {"value": round(world * tasks / secs, 1), "unit": "tasks/s",
            "h2d_bytes_per_step": int(lines[-1]["h2d_bytes"]), "d2h_bytes_per_step": int(lines[-1]["d2h_bytes"]),
            "ms_per_step": round(secs / len(lines) * 1e3, 3), "steps": len(lines), "phases_ms": phases,
            "api": "XKRT C API (xkrt_task_spawn_with_format_with_accesses x tasks, xkrt_task_wait), fresh runtime per step",
            "checksum": lines[-1]["checksum"]}


HEAT_CXX = os.path.join(HERE, "xkaapi_b200", "examples", "heat_cxx")


def _example_lines(exe, argv, local, timeout=900):
    env = dict(os.environ)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = vis.split(",")[local] if vis else str(local)
    r = subprocess.run([exe] + [str(a) for a in argv], env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed: {r.stderr[-400:]}")
    return [json.loads(l) for l in r.stdout.strip().splitlines()]


def config_h_study(local, n=1024, ts=128, steps=100):
    """The plain heat configuration (1024^2 FP64, 128^2 tiles, 100 steps: 6,400 tile tasks), spawn
    -> wait, three ways: the C API with the library's tile body (heat_xkrt), the C++ source API
    with the program's own CUDA kernel launched from its task body (heat_cxx), and the reference's
    host-only runtime on all host threads (oracle/_ref/ref_heat); median of the repetitions after
    a warm-up one."""
    out = {"workload": f"heat {n}^2 FP64, {ts}^2 tiles, {steps} steps ({(n // ts) ** 2 * steps} tasks), spawn -> wait, fresh runtime"}
    try:
        ln = _example_lines(HEAT_XKRT, [n, n, ts, steps, 6], local)[1:]
        out["capi_builtin_body"] = {"tasks_per_s": round(statistics.median(l["tasks_per_s"] for l in ln), 1),
                                    "fused": ln[-1]["fused"], "reps": len(ln)}
    except Exception as ex:
        out["capi_builtin_body"] = {"failed": str(ex)[:300]}
    try:
        ln = _example_lines(HEAT_CXX, [n, n, ts, steps, 4], local)[1:]
        out["cxx_user_body"] = {"tasks_per_s": round(statistics.median(l["tasks_per_s"] for l in ln), 1), "reps": len(ln),
                                "same_result_as_capi": ln[-1]["checksum"] == _example_lines(HEAT_XKRT, [n, n, ts, steps, 1], local)[0]["checksum"]}
    except Exception as ex:
        out["cxx_user_body"] = {"failed": str(ex)[:300]}
    if os.path.exists(REF_HEAT):
        cores = host_threads()
        try:
            vals = [ref_heat_sample(cores, steps, n=n, ts=ts)[0] for _ in range(4)][1:]
            out["reference_cpu"] = {"tasks_per_s": round(statistics.median(vals), 1), "cores": cores,
                                    "what": "the reference's host-only runtime (oracle/_ref/ref_heat), same graph, spawn -> task_wait"}
        except Exception as ex:
            out["reference_cpu"] = {"failed": str(ex)[:300]}
    return out


def user_body_study(local, n=NX, ts=TS, steps=10):
    """The drop-in path of a program that brings its own CUDA tile kernel (examples/heat_cxx: tasks
    built by hand with the C++ source API, kernel launched through task_detachable_kernel_launch,
    run by the host dataflow team) on the headline grid for a few steps; spawn -> wait."""
    try:
        ln = _example_lines(HEAT_CXX, [n, n, ts, steps, 2], local)[1:]
    except Exception as ex:
        return {"failed": str(ex)[:300]}
    return {"tasks": ln[-1]["tasks"], "tasks_per_s": round(ln[-1]["tasks_per_s"], 1), "seconds": round(ln[-1]["seconds"], 3),
            "spawn_s": round(ln[-1]["spawn_s"], 3),
            "workload": f"heat {n}^2 FP64, {ts}^2 tiles, {steps} steps, C++ source API, user CUDA kernel per task; the grids "
                        "placed on the GPU by distribute_async before the timed part, the written blocks copied back to the "
                        "host inside it (at the wait)"}


AXPBY_XKRT = os.path.join(HERE, "xkaapi_b200", "examples", "axpby_xkrt")
REF_AXPBY = os.path.join(HERE, "oracle", "_ref", "ref_axpby")
AXPBY_N, AXPBY_PASSES, AXPBY_SEED, AXPBY_CMIN, AXPBY_CMAX = 1 << 28, 10, 2026, 65536, 16 << 20


def axpby_study(local):
    """axpby task chains (2^28 FP64, 10 passes, seeded chunks of 64 KiB-16 MiB whose boundaries
    move between passes) through the C API with host-resident x and y: one warm-up and one timed
    repetition of spawn -> xkrt_task_wait. Beside it the reference's own host runtime on the same
    graph (same generator) with all host threads."""
    env = dict(os.environ)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = vis.split(",")[local] if vis else str(local)
    args = [str(AXPBY_N), str(AXPBY_PASSES), str(AXPBY_SEED)]
    r = subprocess.run([AXPBY_XKRT] + args + ["2", str(AXPBY_CMIN), str(AXPBY_CMAX)], env=env, capture_output=True,
                       text=True, timeout=900)
    if r.returncode != 0:
        return {"failed": r.stderr[-300:]}
    ln = json.loads(r.stdout.strip().splitlines()[-1])
    dev_bytes = 24.0 * AXPBY_N * AXPBY_PASSES
    out = {"tasks": ln["tasks"], "edges": ln["edges"], "seconds": round(ln["seconds"], 4),
           "tasks_per_s": round(ln["tasks_per_s"], 1),
           "phases_ms": {k: round(ln[k], 1) for k in ("resolve_ms", "coherency_ms", "run_ms", "writeback_ms")},
           "spawn_ms": round(ln["spawn_s"] * 1e3, 1), "h2d_bytes": ln["h2d_bytes"], "d2h_bytes": ln["d2h_bytes"],
           "run_GBps": round(dev_bytes / (ln["run_ms"] / 1e3) / 1e9, 1),
           "workload": f"y = a*x + b*y on 2^28 FP64, {AXPBY_PASSES} passes, chunks log-uniform {AXPBY_CMIN} B-{AXPBY_CMAX >> 20} MiB "
                       "(moving boundaries), segment accesses R x / RW y, host-resident inputs; run_GBps = 24 B x elements x "
                       "passes / run_ms", "checksum": ln["checksum"]}
    if os.path.exists(REF_AXPBY):
        cores = host_threads()
        renv = dict(os.environ, DRIVERS=f"host,{cores}", XKRT_DRIVERS=f"host,{cores}")
        try:
            rl = _ref_run([REF_AXPBY] + args + [str(AXPBY_CMIN), str(AXPBY_CMAX)], renv, timeout=900)
        except Exception as ex:
            rl, out["reference_cpu"] = None, {"failed": str(ex)[:300]}
        if rl:
            out["reference_cpu"] = {"tasks_per_s": rl["tasks_per_s"], "seconds": rl["seconds"], "cores": cores,
                                    "same_result": rl["checksum"] == ln["checksum"],
                                    "what": "the reference's host-only runtime (oracle/_ref/ref_axpby), same graph, spawn -> task_wait"}
    return out


REF_DEPS = os.path.join(HERE, "oracle", "_ref", "ref_deps")
STREAM_MAGIC = 0x314D525453424B58


def ref_deps_time(recs):
    """The reference's own dependency trees (oracle/_ref/ref_deps: KBLASDependencyTree driven by
    task_dependency_resolve, one producer thread as in the reference) on the same stream."""
    if not os.path.exists(REF_DEPS):
        return None
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.bin")
        with open(p, "wb") as f:
            np.array([STREAM_MAGIC, len(recs)], dtype="<u8").tofile(f)
            recs.tofile(f)
        try:
            r = subprocess.run([REF_DEPS, p, os.path.join(d, "o")], capture_output=True, text=True, timeout=300)
        except subprocess.TimeoutExpired:
            return {"failed": "timed out after 300 s"}
    if r.returncode != 0:
        return {"failed": r.stderr[-200:]}
    out = json.loads(r.stdout.strip().splitlines()[-1])
    return {"tasks_per_s": round(out["ntasks"] / out["resolve_s"], 1), "seconds": out["resolve_s"], "cores": 1,
            "unique_edges": out["unique_edges"],
            "what": "the reference's KBLASDependencyTree via task_dependency_resolve on the same stream, one thread"}


def microbench_stream(ntasks, seed, n=8192, ld=8192, align=64, max_units=32, base=1 << 40):
    """Dependency microbench: 1-4 accesses per task on an n x n FP64 matrix (LD = ld), rectangles
    aligned to 64 elements with sides 64*U{1..32}, modes R 60% / W 20% / RW 20%."""
    import xkaapi_b200 as xk
    rng = np.random.default_rng(seed)
    na = rng.integers(1, 5, ntasks)
    tot = int(na.sum())
    units = n // align
    mu = rng.integers(1, max_units + 1, tot); nu = rng.integers(1, max_units + 1, tot)
    xu = (rng.random(tot) * (units - mu + 1)).astype(np.int64); yu = (rng.random(tot) * (units - nu + 1)).astype(np.int64)
    r = rng.integers(0, 10, tot)
    recs = np.zeros(tot, dtype=xk.heat.ACCESS_REC)
    recs["task"] = np.repeat(np.arange(ntasks, dtype=np.uint32), na)
    recs["type"] = 2; recs["mode"] = np.where(r < 6, 1, np.where(r < 8, 2, 3))
    recs["addr"] = base; recs["ld"] = ld; recs["sizeof_type"] = 8
    recs["offset_m"] = xu * align; recs["offset_n"] = yu * align; recs["m"] = mu * align; recs["n"] = nu * align
    return recs


def resolver_microbench(xk, torch, stream, recs, hbm_peak, reps=3):
    """The dependency microbench through the GPU resolver: a fresh resolver's first add + graph
    (its working buffers allocated inside the timing), then the same resolver reset and reused,
    as the runtime keeps its resolver between waits (best of `reps`). Returns (line, edges)."""
    r3 = xk.Resolver(stream)
    t0 = time.perf_counter(); r3.add(recs); g3 = r3.graph(); torch.cuda.synchronize()
    dt_first = time.perf_counter() - t0
    nfirst = int(g3.nedges)
    dts = []
    for _ in range(reps):
        r3.reset()
        t0 = time.perf_counter(); r3.add(recs); g3 = r3.graph(); torch.cuda.synchronize()
        dts.append(time.perf_counter() - t0)
    dt = min(dts) if dts else dt_first
    phases = r3.timing()
    nedges = int(g3.nedges)
    r3.close()
    ntasks = int(recs["task"].max()) + 1
    visits = int(((recs["m"] // 64) * (recs["n"] // 64)).sum())          # 64 x 64-element cells per access
    mb_bytes = 32.0 * len(recs) + 8.0 * nedges + 16.0 * visits
    line = {"tasks": ntasks, "accesses": int(len(recs)), "unique_edges": nedges,
            "seconds": round(dt, 4), "tasks_per_s": round(ntasks / dt),
            "seconds_fresh_resolver": round(dt_first, 4),
            "same_edges_fresh_and_reused": nfirst == nedges,
            "phases_ms": {"host_ops": round(phases[0], 2), "compress": round(phases[1], 2),
                          "batch_device": round(phases[2], 2)},
            "timing": "wall time of add + graph on a reset, reused resolver (best of %d); "
                      "seconds_fresh_resolver: the first add + graph of a new resolver" % reps,
            "roofline": {"bound": "hbm", "achieved": round(mb_bytes / dt / 1e9, 2), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(mb_bytes / dt / 1e9 / hbm_peak, 5),
                         "algorithmic_bytes": mb_bytes, "cell_visits": visits,
                         "what": "32 B per access + 8 B per unique edge + 16 B per visit of a "
                                 "64 x 64-element cell, over the wall time of add + graph"}}
    return line, nedges


def serve_trace(ngraphs, seed, ts=128):
    """Served-stream trace: grid side log-uniform in [256, 8192] rounded to a multiple of the
    tile; steps uniform in {10..200}; FP64 / FP32 storage 50/50; Poisson arrival order."""
    rng = np.random.default_rng(seed)
    side = np.exp(rng.uniform(np.log(256), np.log(8192), ngraphs))
    side = np.clip((np.round(side / ts) * ts).astype(np.int64), ts * 2, 8192)
    steps = rng.integers(10, 201, ngraphs)
    f32 = rng.integers(0, 2, ngraphs)
    gaps = rng.exponential(1.0, ngraphs)              # unit-rate Poisson process, scaled later
    bytes_ = (side.astype(np.float64) - 2) ** 2 * steps * np.where(f32 == 1, 8.0, 16.0)
    return side, steps, f32, np.cumsum(gaps), bytes_


_SERVE_IO = {}


def serve_io(torch):
    """Page-locked host buffers every served request reads its initial grid from and writes its
    result to: one input of the largest grid (seeded U[0,1) values; a request takes its first
    nx*ny elements) and one result buffer that concurrent results overwrite (only the time of
    the transfers matters here; the parity tests check results)."""
    if not _SERVE_IO:
        n = 8192 * 8192
        inp = torch.empty(n, dtype=torch.float64).pin_memory()
        inp.numpy()[:] = np.random.default_rng(SEED).random(n)
        _SERVE_IO["in"] = inp
        _SERVE_IO["out"] = torch.empty(n, dtype=torch.float64).pin_memory()
    return _SERVE_IO["in"].data_ptr(), _SERVE_IO["out"].data_ptr()


def serve_tiles(side, policy):
    """Tile side of each served graph: 128 ("128"), or 256 for grids of 2048 and more, whose
    128^2 tiles would be 256 or more per step ("256from2048"); the trace fixes the graphs, the
    runtime chooses their tiling (the batched configuration tunes the tile over 128-1024)."""
    side = np.asarray(side)
    if policy == "256from2048":
        return np.where(side >= 2048, 256, 128)
    return np.full(len(side), 128)


def serve_requests(xk, side, steps, f32, arrivals, io=None, tiles=None):
    reqs = (xk.Request * len(side))()
    tiles = np.full(len(side), 128) if tiles is None else tiles
    for k, r in enumerate(reqs):
        r.arrival_s, r.nx, r.ny, r.ts, r.steps, r.f32 = (float(arrivals[k]), int(side[k]), int(side[k]), int(tiles[k]),
                                                         int(steps[k]), int(f32[k]))
        r.seed, r.c = 7000 + k, COEF
        r.input, r.result = (io if io else (None, None))
    return reqs


def serve_study(xk, torch, ngraphs=2000, slots=16, load=0.8):
    side, steps, f32, unit_arrivals, bytes_ = serve_trace(ngraphs, 2026)
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(150e9, free - 8e9))
    io = serve_io(torch)
    srv = xk.Server(budget_bytes=budget, slots=slots)
    # capacity: the first graphs of the trace all arriving at once (closed loop), measured on the
    # second pass, after the first has resolved the periodic graph of every shape they use; the
    # same with one persistent launch per request (the former serving loop) for comparison
    cal = min(300, ngraphs)
    for _ in range(2):
        reqs = serve_requests(xk, side[:cal], steps[:cal], f32[:cal], np.zeros(cal), io)
        srv.run(reqs)
    capacity = float(bytes_[:cal].sum()) / max(r.finish_s for r in reqs)          # bytes/s served
    os.environ["XKB_SERVE_MODE"] = "launch"
    try:
        reqs = serve_requests(xk, side[:cal], steps[:cal], f32[:cal], np.zeros(cal), io)
        srv.run(reqs)
        capacity_launch = float(bytes_[:cal].sum()) / max(r.finish_s for r in reqs)
    finally:
        del os.environ["XKB_SERVE_MODE"]
    # the trace: Poisson arrivals whose offered HBM traffic is `load` x the capacity
    rate = load * capacity / float(bytes_.mean())                                  # graphs/s
    arrivals = unit_arrivals / rate
    reqs = serve_requests(xk, side, steps, f32, arrivals, io)
    t0 = time.perf_counter()
    srv.run(reqs)
    wall = time.perf_counter() - t0
    srv.close()
    lat = np.array([r.finish_s - r.arrival_s for r in reqs]) * 1e3
    wait = np.array([r.start_s - r.arrival_s for r in reqs]) * 1e3
    fin = max(r.finish_s for r in reqs)
    tasks = int(sum((-(-int(side[k]) // 128)) ** 2 * int(steps[k]) for k in range(ngraphs)))
    return {"graphs": ngraphs, "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "mean_ms": round(float(lat.mean()), 3),
            "admission_wait_p99_ms": round(float(np.percentile(wait, 99)), 3),
            "tasks": tasks, "tasks_per_s": round(tasks / fin), "GBps": round(float(bytes_.sum()) / fin / 1e9, 1),
            "capacity_GBps": round(capacity / 1e9, 1), "capacity_frac": round(capacity / 1e9 / peaks()[0], 3),
            "capacity_launch_mode_GBps": round(capacity_launch / 1e9, 1), "offered_load": load,
            "rate_graphs_per_s": round(rate, 1),
            "span_s": round(float(arrivals[-1]), 3), "makespan_s": round(fin, 3), "wall_s": round(wall, 3),
            "budget_GB": round(budget / 1e9, 1), "slots": slots,
            "trace": "Poisson arrivals, side log-uniform 256-8192 (multiple of 128), steps U{10..200}, FP64/FP32 50/50, "
                     "128^2 tiles; load calibrated on a closed-loop run of the first 300 graphs (second pass, shapes resolved)",
            "latency": "arrival -> result in host memory: the input grid copied in from page-locked host memory at "
                       "admission and the result copied out are inside it",
            "loop": "one persistent kernel for the whole trace runs every admitted request's tile tasks"}


def run_study(args):
    """One study alone on cuda:0, its JSON line on stdout (no headline, no CPU baseline)."""
    import torch
    import xkaapi_b200 as xk
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    hbm_peak, _ = peaks()
    if args.study == "resolver":
        recs = microbench_stream(args.tasks, 12345)
        line, _ = resolver_microbench(xk, torch, stream, recs, hbm_peak, reps=args.steps)
        print(json.dumps({"study": "resolver", **line}), flush=True)
        return 0
    if args.study == "graph":
        n, steps, esz = NX, STEPS, (4 if args.f32 else 8)
        g = torch.rand((n, n), dtype=torch.float64, generator=torch.Generator().manual_seed(SEED))
        g[0, :] = 0; g[-1, :] = 0; g[:, 0] = 0; g[:, -1] = 0
        a = g.to(device="cuda", dtype=torch.float32 if args.f32 else torch.float64); b = a.clone()
        del g
        res, graph, _ = build_heat_graph(xk, torch, a, b, n, n, args.tile, steps, stream, esize=esz)
        d = xk.heat_task_descs((a.data_ptr(), b.data_ptr()), n, n, n, args.tile, args.tile, steps, COEF, f32=args.f32)
        sch = xk.Scheduler(stream); sch.set_team(args.team); sch.set_tasks(d); del d
        if args.prefetch:
            sch.set_prefetch(args.prefetch)
        runs = []
        for k in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                sch.run(graph); sch.wait()
            if k >= args.warmup:
                runs.append(sch.kernel_ms())
        best = min(runs)
        print(json.dumps({"study": "graph", "size": n, "steps": steps, "dtype": "f32" if args.f32 else "f64",
                          "tile": args.tile, "warps_per_task": args.team,
                          "tasks": int(graph.ntasks), "kernel_ms": [round(x, 3) for x in runs],
                          "GBps_best": round(2.0 * esz * cells_all(n, n) * steps / (best / 1e3) / 1e9, 1)}), flush=True)
        sch.close(); res.close()
        return 0
    # serve: closed-loop capacity of a few shapes, device loop and one launch per request
    io = serve_io(torch)
    free, _ = torch.cuda.mem_get_info()
    srv = xk.Server(budget_bytes=int(min(150e9, free - 8e9)), slots=args.slots)
    side, steps, f32, _, _ = serve_trace(2000, 2026)
    cases = {"8 x 4096^2 FP64 x 100 steps": (np.full(8, 4096), np.full(8, 100), np.zeros(8, np.int64)),
             "first 300 graphs of the trace": (side[:300], steps[:300], f32[:300])}
    for name, (sd, st, f) in cases.items():
        nbytes = float(((sd.astype(np.float64) - 2) ** 2 * st * np.where(f == 1, 8.0, 16.0)).sum())
        for mode, withio, policy in (("device", True, "128"), ("device", True, "256from2048"), ("device", False, "128"),
                                     ("launch", True, "128"), ("launch", False, "128")):
            if mode == "launch":
                os.environ["XKB_SERVE_MODE"] = "launch"
            else:
                os.environ.pop("XKB_SERVE_MODE", None)
            for _ in range(2):          # the second pass: every shape's graph already resolved
                reqs = serve_requests(xk, sd, st, f, np.zeros(len(sd)), io if withio else None, serve_tiles(sd, policy))
                srv.run(reqs)
            fin = max(r.finish_s for r in reqs)
            print(json.dumps({"study": "serve", "case": name, "mode": mode, "host_io": withio, "tiles": policy,
                              "GBps": round(nbytes / fin / 1e9, 1), "makespan_s": round(fin, 3),
                              "p50_ms": round(float(np.percentile([(r.finish_s - r.start_s) * 1e3 for r in reqs], 50)), 2)}),
                  flush=True)
    os.environ.pop("XKB_SERVE_MODE", None)
    srv.close()
    return 0


def main():
    global NX, NY, STEPS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="smaller side studies (plain/graph/microbench)")
    ap.add_argument("--no-side", action="store_true",
                    help="run only the headline measurement (no forms / stencil / resolver / CPU side studies)")
    ap.add_argument("--size", type=int, default=NX, help="grid side (default 16384)")
    ap.add_argument("--graph-steps", type=int, default=STEPS, help="Jacobi steps in the graph (default 500)")
    ap.add_argument("--study", choices=["resolver", "graph", "serve"],
                    help="run one study alone and print its JSON (the commands of the profile summaries): "
                         "resolver = the dependency microbench (--tasks); graph = the heat graph on the "
                         "persistent scheduler (--size, --graph-steps, --f32, --prefetch, --steps); "
                         "serve = serving capacity with and without host I/O, device loop and one launch per request")
    ap.add_argument("--tasks", type=int, default=65536, help="--study resolver: tasks of the microbench")
    ap.add_argument("--f32", action="store_true", help="--study graph: FP32 storage")
    ap.add_argument("--prefetch", type=int, default=0, help="--study graph: L2 prefetch distance (0: the default)")
    ap.add_argument("--slots", type=int, default=16, help="served stream: requests on the device at once")
    ap.add_argument("--tile", type=int, default=TS, help="--study graph: tile side")
    ap.add_argument("--team", type=int, default=1, help="--study graph: warps per task (1, 2, 4, 8)")
    args = ap.parse_args()
    NX = NY = args.size
    STEPS = args.graph_steps
    if args.impl == "reference":
        return run_reference(args)
    if args.study:
        return run_study(args)

    import torch
    import xkaapi_b200 as xk
    rank, world, local = dist_setup(args.gpus)
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    hbm_peak, peak_kind = peaks()
    extra = {}

    # ---------------- resolver microbench, first: a latency-bound kernel chain that a GPU held
    # at its power cap by the stencil runs below would time at a lower clock ----------------
    mb = None
    if rank == 0 and not args.no_side:
        mb_tasks = 16384 if args.quick else 65536
        mb_recs = microbench_stream(mb_tasks, 12345)
        mb = resolver_microbench(xk, torch, stream, mb_recs, hbm_peak, reps=5)
        mb[0]["when"] = "before the heat studies (idle GPU, boost clocks)"

    # ---------------- headline: persistent scheduler over the whole 500-step graph ----------
    host = torch.empty((NY, NX), dtype=torch.float64).pin_memory()
    rng = np.random.default_rng(SEED + rank)
    hv = host.numpy()
    hv[:] = 0.0
    hv[1:NY - 1, 1:NX - 1] = rng.random((NY - 2, NX - 2))
    a = torch.empty((NY, NX), dtype=torch.float64, device="cuda")
    b = torch.empty_like(a)
    a.copy_(host); b.copy_(a)
    torch.cuda.synchronize()
    res, graph, t_resolve = build_heat_graph(xk, torch, a, b, NX, NY, TS, STEPS, stream)
    ntasks = graph.ntasks
    descs = xk.heat_task_descs((a.data_ptr(), b.data_ptr()), NX, NY, NX, TS, TS, STEPS, COEF)
    sch = xk.Scheduler(stream)
    sch.set_tasks(descs)
    del descs
    extra["graph_build"] = {"tasks": int(ntasks), "edges": int(graph.nedges), "resolve_s": round(t_resolve, 3),
                            "resolve_tasks_per_s": round(ntasks / t_resolve)}

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            sch.run(graph); sch.wait()
    barrier(world); torch.cuda.synchronize()
    clocks = Clocks(dev); clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    run_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.nvtx.range_push("timed")
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k in range(args.steps):
            run_ev[k][0].record(stream)
            sch.run(graph)
            run_ev[k][1].record(stream)
        e1.record(stream)
    stream.synchronize()
    torch.cuda.nvtx.range_pop()
    runs_ms = [round(x.elapsed_time(y), 3) for x, y in run_ev]
    ms_total = e0.elapsed_time(e1)
    clk = clocks.stop()
    executed = sch.wait()
    last_kernel_ms = sch.kernel_ms()
    barrier(world)
    ms_total = max_over_ranks(ms_total, world)
    ms_step = ms_total / args.steps
    value = world * ntasks * args.steps / (ms_total / 1e3)
    assert executed == ntasks, (executed, ntasks)
    cells = (NX - 2) * (NY - 2)
    alg_bytes = 16.0 * cells * STEPS
    achieved = alg_bytes / (last_kernel_ms / 1e3) / 1e9
    traffic = profile_traffic() if (NX, STEPS) == (16384, 500) else None

    # result check against the CPU restatement on a sample of rows after one more run is not
    # possible at this size; the parity suite covers correctness. Keep a checksum instead.
    res_grid = a if STEPS % 2 == 0 else b
    checksum = float(res_grid.sum().item())
    # FP64 checks of the last step: the other grid holds the state one step earlier
    extra["checks_fp64"] = {"f64": xk.heat_norms(b if STEPS % 2 == 0 else a, res_grid, NX, NY, NX, COEF, stream=stream),
                            "what": "xkb_heat_norms on the last Jacobi step of the graph: boundary max |g| (Dirichlet 0), "
                                    "interior L2 norm, residual max |dst - update(src)| with the update in FP64"}

    # ---------------- e2e replay: the resolved graph re-run with host grids copied in and out --
    torch.cuda.synchronize()
    out_host = torch.empty_like(host).pin_memory()
    with torch.cuda.stream(stream):
        sch.run(graph); sch.wait()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        f0.record(stream)
        for _ in range(args.steps):
            a.copy_(host, non_blocking=True)
            b.copy_(a, non_blocking=True)
            sch.run(graph)
            out_host.copy_(res_grid, non_blocking=True)
        f1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), world)
    e2e_value = world * ntasks * args.steps / (e2e_ms / 1e3)
    bytes_grid = NX * NY * 8

    # ---------------- FP32 storage: the same graph on FP32 grids, error vs the FP64 run --------
    # the last replay step ran the whole graph from the initial grid: res_grid holds FP64 after
    # STEPS steps (bit-exact with the oracle by the parity tests)
    if rank == 0 and not args.no_side:
        a32 = host.to(device="cuda", dtype=torch.float32); b32 = a32.clone()
        res32, g32, t32 = build_heat_graph(xk, torch, a32, b32, NX, NY, TS, STEPS, stream, esize=4)
        d32 = xk.heat_task_descs((a32.data_ptr(), b32.data_ptr()), NX, NY, NX, TS, TS, STEPS, COEF, f32=True)
        s32 = xk.Scheduler(stream); s32.set_team(1); s32.set_tasks(d32); del d32   # one warp per FP32 tile
        with torch.cuda.stream(stream):
            s32.run(g32); s32.wait()
        extra["checks_fp64"]["f32"] = xk.heat_norms(b32 if STEPS % 2 == 0 else a32, a32 if STEPS % 2 == 0 else b32,
                                                    NX, NY, NX, COEF, stream=stream)
        out32 = (a32 if STEPS % 2 == 0 else b32).double()
        err32 = float((out32 - res_grid).abs().max().item()) / float(res_grid.abs().max().item())
        del out32
        ms32 = []
        for _ in range(2):
            with torch.cuda.stream(stream):
                s32.run(g32); s32.wait()
            ms32.append(s32.kernel_ms())
        best = min(ms32)
        extra["graph_f32"] = {"tasks": int(g32.ntasks), "kernel_ms": round(best, 3), "tasks_per_s": round(g32.ntasks / (best / 1e3)),
                              "GBps": round(8.0 * cells_all(NX, NY) * STEPS / (best / 1e3) / 1e9, 1),
                              "max_rel_error_vs_f64": err32,
                              "error_check": f"FP32-storage graph vs the FP64 graph, both {STEPS} steps from the same initial grid "
                                             "(max abs difference / max |FP64|); tolerance 1e-5",
                              "resolve_s": round(t32, 3),
                              "frac": round(8.0 * cells_all(NX, NY) * STEPS / (best / 1e3) / 1e9 / hbm_peak, 3)}
        s32.close(); res32.close()
        # the batched config autotunes the tile (128-1024) and the warps per task: the FP32 graph
        # at the tuned shape, the whole STEPS-step graph from the same grids
        from xkaapi_b200.autotune import autotune_heat
        a32.copy_(host); b32.copy_(a32)
        best32, cands32 = autotune_heat(a32, b32, NX, NY, steps=4, f32=True, stream=stream)
        a32.copy_(host); b32.copy_(a32)
        tile32 = best32["tile"]
        rt, gt, tt = build_heat_graph(xk, torch, a32, b32, NX, NY, tile32, STEPS, stream, esize=4)
        dt32 = xk.heat_task_descs((a32.data_ptr(), b32.data_ptr()), NX, NY, NX, tile32, tile32, STEPS, COEF, f32=True)
        st32 = xk.Scheduler(stream); st32.set_team(best32["team"]); st32.set_tasks(dt32); del dt32
        with torch.cuda.stream(stream):
            st32.run(gt); st32.wait()                   # from the initial grid: the error check
        outt = (a32 if STEPS % 2 == 0 else b32).double()
        errt = float((outt - res_grid).abs().max().item()) / float(res_grid.abs().max().item())
        del outt
        mst = []
        for _ in range(2):
            with torch.cuda.stream(stream):
                st32.run(gt); st32.wait()
            mst.append(st32.kernel_ms())
        bt = min(mst)
        gbt = 8.0 * cells_all(NX, NY) * STEPS / (bt / 1e3) / 1e9
        extra["graph_f32_tuned"] = {"tile": tile32, "warps_per_task": best32["team"], "tasks": int(gt.ntasks),
                                    "kernel_ms": round(bt, 3), "GBps": round(gbt, 1), "frac": round(gbt / hbm_peak, 3),
                                    "max_rel_error_vs_f64": errt, "autotune_candidates": len(cands32),
                                    "what": f"the {STEPS}-step FP32-storage graph at the tile and warps per task the "
                                            "autotuner picked on a 4-step graph of the same grids (the batched "
                                            "config tunes the tile over 128-1024)"}
        st32.close(); rt.close(); del a32, b32
        torch.cuda.empty_cache()

    # ---------------- forms at equal work: first two steps ------------------------------------
    forms = {}
    if rank == 0 and not args.no_side:
        win = 2
        res2, g2, _ = build_heat_graph(xk, torch, a, b, NX, NY, TS, win, stream)
        d2 = xk.heat_task_descs((a.data_ptr(), b.data_ptr()), NX, NY, NX, TS, TS, win, COEF)
        s2 = xk.Scheduler(stream)
        s2.set_tasks(d2)
        for name, form, reps in (("persistent", xk.FORM_PERSISTENT, 10), ("plain", xk.FORM_PLAIN, 2),
                                 ("cuda_graph", xk.FORM_GRAPH, 5)):
            t_build = time.perf_counter()
            with torch.cuda.stream(stream):
                s2.run(g2, form); s2.wait()
            t_build = time.perf_counter() - t_build
            h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                h0.record(stream)
                for _ in range(reps):
                    s2.run(g2, form)
                h1.record(stream)
            stream.synchronize(); s2.wait()
            ms = h0.elapsed_time(h1) / reps
            forms[name] = {"tasks": int(g2.ntasks), "ms": round(ms, 3), "tasks_per_s": round(g2.ntasks / (ms / 1e3)),
                           "first_run_s": round(t_build, 3)}
        forms["fused_vs_plain"] = round(forms["persistent"]["tasks_per_s"] / forms["plain"]["tasks_per_s"], 2)
        forms["graph_vs_plain"] = round(forms["cuda_graph"]["tasks_per_s"] / forms["plain"]["tasks_per_s"], 2)
        s2.close(); res2.close()

        # whole-step stencil kernel (all tile tasks of a step fused into one launch)
        sten = {}
        start = a.clone()
        finals = {}
        for dt, name, esz in ((torch.float64, "f64", 8), (torch.float32, "f32", 4)):
            x = start.clone() if dt == torch.float64 else start.float()
            y = torch.empty_like(x); y.copy_(x)
            with torch.cuda.stream(stream):
                for _ in range(3):
                    xk.heat_step(x, y, NX, NY, NX, COEF, stream=stream); x, y = y, x
                q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                q0.record(stream)
                for _ in range(10):
                    xk.heat_step(x, y, NX, NY, NX, COEF, stream=stream); x, y = y, x
                q1.record(stream)
            stream.synchronize()
            ms = q0.elapsed_time(q1) / 10
            gbs = 2.0 * esz * cells / (ms / 1e3) / 1e9
            sten[name] = {"ms_per_step": round(ms, 4), "GBps": round(gbs, 1), "frac_of_peak": round(gbs / hbm_peak, 3)}
            finals[name] = x
            del y
        # FP32-storage error of this run: the FP32 grid after the same 13 steps against the FP64
        # grid (the FP64 kernel is bit-exact with the oracle), max abs error over max |FP64|
        ref64 = finals["f64"]
        err = float((finals["f32"].double() - ref64).abs().max().item()) / float(ref64.abs().max().item())
        sten["f32_max_rel_error_vs_f64"] = err
        sten["f32_error_check"] = "13 Jacobi steps of the 16384^2 grid from the same start; tolerance 1e-5"
        del finals, ref64, start
        extra["stencil_whole_step"] = sten

        # autotuner: tile shape x warps per task on a short graph of the same grid
        from xkaapi_b200.autotune import autotune_heat
        best, cands = autotune_heat(a, b, NX, NY, steps=4, stream=stream)
        extra["autotune"] = {"best": best, "candidates": len(cands),
                             "tile128_best": max((r for r in cands if r["tile"] == 128), key=lambda r: r["GBps"])}

        # resolver microbench (measured first), beside the reference's trees on the same stream
        recs = mb_recs
        extra["resolver_microbench"], nedges = mb
        ref = ref_deps_time(recs)
        if ref:
            ref["same_unique_edges"] = ref.pop("unique_edges") == nedges
            extra["resolver_microbench"]["reference_cpu"] = ref

    # ---------------- served stream (after releasing the headline graph's memory) -----------
    sch.close(); res.close()
    del a, b
    torch.cuda.synchronize(); torch.cuda.empty_cache()

    # ---------------- e2e: the drop-in C API, spawn -> wait, resolution included ------------
    e2e = capi_e2e(max(2, min(args.steps, 3)), world, local)
    if rank == 0 and not args.no_side:
        extra["config_h"] = config_h_study(local)
        extra["e2e_user_body"] = user_body_study(local)
        extra["axpby_chains"] = axpby_study(local)
    if rank == 0 and not args.no_side:
        extra["serve"] = serve_study(xk, torch, ngraphs=400 if args.quick else 2000, slots=args.slots)

    # ---------------- CPU baseline (rank 0, N=1) ----------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_side:
        cpu = cpu_baseline_sample(10.0)

    if rank == 0:
        line = {
            "metric": "tasks/s", "value": round(value, 1), "unit": "tasks/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded U[0,1) interior, Dirichlet 0 boundary)",
            "config": {"workload": f"batched heat-diffusion-2d: {NX}x{NY} FP64 grid, {TS}x{TS} tile tasks, {STEPS} steps "
                                   f"({ntasks} tasks per bench step), dependencies from the GPU resolver, persistent "
                                   "device scheduler", "l2": "inputs (2 grids of 8*NX*NY bytes) larger than L2",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(achieved / hbm_peak, 3), "traffic": traffic,
                         "kernel": "sched_persistent_kernel", "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": round(last_kernel_ms, 3)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_replay": {"value": round(e2e_value, 1), "unit": "tasks/s", "h2d_bytes_per_step": bytes_grid,
                           "d2h_bytes_per_step": bytes_grid, "ms_per_step": round(e2e_ms / args.steps, 3),
                           "what": "the resolved graph re-run by xkb_sched_run, the grid copied in from pinned host memory "
                                   "and the result copied out every step"},
            "gpu_launches": 3 * args.steps,
            "clocks": clk,
            "forms_first_2_steps": forms,
            "runs_ms": runs_ms,
            "checksum": checksum,
        }
        line.update(extra)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
