"""Regenerates tests/golden/deps_golden.npz from the REFERENCE's own dependency trees and
tests/golden/plan_golden.npz from the reference's own coherency controller (memory tree).

Each case is a seeded access stream (tests/streams.py) run through oracle/_ref/ref_deps,
which drives the reference's KBLASDependencyTree / IntervalDependencyTree via
src/task/task.cc:task_dependency_resolve (built by oracle/ref/build_ref.sh). The stream
records and the reference's unique (pred, succ) task pairs are stored side by side, so the
fixtures pin the oracle restatement and the GPU resolver without the reference present.

Known-answer cases restate the reference's own ordering tests:
  tests/task-dependency-interval.cc:86-121         W/R/RW chain on overlapping intervals
  tests/task-dependency-interval-matrix.cc:84-160  interval W -> matrix W -> interval W
Plan fixtures: oracle/_ref/ref_plan drives KBLASMemoryTree::fetch
(include/xkrt/memory/access/blas/memory-tree.hpp:1805-1874) under the canonical schedule (fetches in
spawn order, each fetch's copies completed before the next); allocations, device views and the
sorted copy records are stored.
axpby fixtures: oracle/_ref/ref_axpby (the reference's host-only runtime running the seeded
axpby task chains with segment accesses, oracle/ref/ref_axpby.cc); the final y of each case is
stored with its parameters, pinning the oracle's restatement of the chain generator and update.
wrap fixtures: streams with matrix tiles that wrap the leading dimension (tests/streams.py
mixed_stream), where the reference's dependency tree is not point-wise
(include/xkrt/memory/access/blas/dependency-tree.hpp:228-256 applies a PUT to whole split-off
nodes that meet the access's other rect): the reference's edges and the point-wise edges of the
oracle restatement (oracle/_bin/deps_oracle) are both stored, so the exact difference is pinned.
register fixtures: ref_plan with registration events (the reference's default build splits its
trees at registered pages, memory-tree.hpp:2184-2240); each case's plan is stored with the
plan of the same stream without registrations so the splits' effect is visible.
Run: python tests/golden/make_golden.py [deps] [plan] [axpby] [wrap] [register]   (default: all; needs the
binaries of oracle/ref/build_ref.sh and oracle/Makefile)
"""
import os, subprocess, sys, tempfile
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
import streams as S  # noqa: E402


def ref_edges(recs):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.bin")
        S.write_stream(p, recs)
        subprocess.run([os.path.join(REPO, "oracle/_ref/ref_deps"), p, os.path.join(d, "o")],
                       check=True, capture_output=True)
        return S.read_edges(os.path.join(d, "o.edges"))


def mixed(kind, seed, n=60):
    """Small random streams: matrices of one (ld, sizeof) without LD wrap-around, segments,
    all access modes. Kinds: 'mat', 'seg', 'segmat'."""
    rng = np.random.default_rng(seed)
    modes = [S.R, S.W, S.RW, S.R | S.V, S.W | S.V, S.R | S.D]
    rows = []
    for t in range(n):
        for _ in range(int(rng.integers(1, 4))):
            mode = modes[int(rng.integers(0, len(modes)))]
            seg = kind == "seg" or (kind == "segmat" and rng.integers(0, 2) == 1)
            if seg:
                a = 4096 + int(rng.integers(0, 2048)); b = a + int(rng.integers(1, 600))
                rows.append((t, S.SEGMENT, mode, 0, a, b, 0, 0, 0, 0, 0))
            else:
                m = int(rng.integers(1, 33)); om = int(rng.integers(0, 64 - m + 1))
                n_ = int(rng.integers(1, 9)); on = int(rng.integers(0, 16))
                rows.append((t, S.MATRIX, mode, 0, 4096, 64, om, on, m, n_, 8))
    return np.array(rows, dtype=S.REC)


def handle_mixed(seed, n=80):
    """Handle accesses (a few handles, every mode incl. VR/VW/D) mixed with segments and
    matrices whose addresses reuse the handle values: handles live in their own domain."""
    rng = np.random.default_rng(seed)
    modes = [S.R, S.W, S.RW, S.R | S.V, S.W | S.V, S.D, S.R | S.D]
    handles = [4096, 4100, 0x7000, 12345]
    rows = []
    for t in range(n):
        for _ in range(int(rng.integers(1, 4))):
            mode = modes[int(rng.integers(0, len(modes)))]
            k = int(rng.integers(0, 3))
            if k == 0:
                rows.append((t, S.HANDLE, mode, 0, handles[int(rng.integers(0, len(handles)))], 0, 0, 0, 0, 0, 0))
            elif k == 1:
                a = 4096 + int(rng.integers(0, 64)); rows.append((t, S.SEGMENT, mode, 0, a, a + int(rng.integers(1, 40)), 0, 0, 0, 0, 0))
            else:
                m = int(rng.integers(1, 9)); om = int(rng.integers(0, 16 - m + 1))
                rows.append((t, S.MATRIX, mode, 0, 4096, 16, om, int(rng.integers(0, 4)), m, int(rng.integers(1, 4)), 8))
    return np.array(rows, dtype=S.REC)


def handle_diagrams():
    """The handle map's two diagrams on one handle (dependency-map.hpp:200-223, :247-262):
    W; 4 concurrent W; 3 R (an extra writer before the first); 2 concurrent W (an extra writer
    before the first); W."""
    ops = [S.W, "c", "c", "c", "c", S.R, S.R, S.R, "c", "c", S.W]
    rows = [(t, S.HANDLE, S.W if o == "c" else o, (4 if o == "c" else 1) << 8, 0x5000, 0, 0, 0, 0, 0, 0)
            for t, o in enumerate(ops)]
    return np.array(rows, dtype=S.REC)


def cases():
    H = 0x5000
    # restates tests/task-dependency-handle.cc:86-119 (W, R, RW on one handle: T0 -> T1 -> T2)
    yield "ref_handle_chain", S.from_tuples([[("h", S.W, H)], [("h", S.R, H)], [("h", S.RW, H)]])
    for seed in range(3):
        yield f"handle_mixed_{seed}", handle_mixed(seed + 50)
    yield "handle_concurrent_diagrams", handle_diagrams()
    for seed in range(4):
        yield f"handle_concurrent_{seed}", S.handle_concurrent_stream(seed + 70)
    X = 0x10000
    yield "ref_interval_chain", S.from_tuples([[("s", S.W, X - 64, X + 64)],
                                              [("s", S.R, X, X + 76)],
                                              [("s", S.RW, X - 12, X + 48)]])
    yield "ref_interval_matrix_chain", S.from_tuples([[("s", S.W, 0, 100)],
                                                     [("m", S.W, 3, 8, 0, 0, 8, 8, 1)],
                                                     [("s", S.W, 0, 100)]])
    yield "heat_64_t16_s4", S.heat_stream(64, 64, 16, 16, 4)
    yield "heat_1024_t128_s3", S.heat_stream(1024, 1024, 128, 128, 3)
    yield "heat_200x136_t64x48_s3", S.heat_stream(200, 136, 64, 48, 3)
    yield "microbench_1024_2000", S.microbench_stream(2000, 7, n=1024, ld=1024)
    # grids not aligned to ld*sizeof: every tile wraps the leading dimension in the address frame
    yield "heat_1024_t128_s3_unaligned", S.heat_stream(1024, 1024, 128, 128, 3, base_src=(1 << 20) + 4096,
                                                       base_dst=(1 << 24) + 8)
    for kind in ("mat", "seg", "segmat"):
        for seed in range(3):
            yield f"mixed_{kind}_{seed}", mixed(kind, seed)


def ref_plan(recs):
    """The reference memory tree's plan (oracle/_ref/ref_plan), canonical schedule. Copy records
    are sorted (a task's copies have no order among themselves in the reference's fetch list)."""
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.bin")
        S.write_stream(p, recs)
        subprocess.run([os.path.join(REPO, "oracle/_ref/ref_plan"), p, os.path.join(d, "o")],
                       check=True, capture_output=True)
        plan = np.fromfile(os.path.join(d, "o.plan"), dtype="<i8").reshape(-1, 14)
        allocs = np.fromfile(os.path.join(d, "o.allocs"), dtype="<i8")
        views = np.fromfile(os.path.join(d, "o.views"), dtype="<i8").reshape(-1, 5)
    if len(plan):
        plan = plan[np.lexsort(tuple(plan[:, k] for k in range(13, -1, -1)))]
    return plan, allocs, views


def plan_cases():
    """Streams for the transfer-plan fixtures. Record field `reserved` bit 0 = fetch to the host."""
    heat = S.heat_stream(1024, 1024, 128, 128, 4, base_src=1 << 30, base_dst=(1 << 30) + (1 << 24))
    yield "plan_heat_1024_t128_s4", heat
    small = S.heat_stream(256, 256, 64, 64, 5, base_src=1 << 20, base_dst=1 << 21)
    export = S.from_tuples([[("m", S.R, 1 << 21, 256, 0, 0, 256, 256, 8)]])
    export["task"] = small["task"].max() + 1
    export["reserved"] = 1
    yield "plan_heat_256_export", np.concatenate([small, export])
    for seed in range(4):
        recs = S.microbench_stream(7, seed, n=256, ld=256, align=16, max_side_units=6)
        rng = np.random.default_rng(seed + 1000)
        recs["reserved"] = (rng.random(len(recs)) < 0.25).astype(np.uint16)
        yield f"plan_mat_wb_{seed}", recs
    # bases not aligned to ld*sizeof: tiles wrap the leading dimension in the address frame
    yield "plan_heat_256_unaligned", S.heat_stream(256, 256, 64, 64, 4, base_src=(1 << 20) + 1024, base_dst=(1 << 22) + 512)
    for seed in range(3):
        rng = np.random.default_rng(seed)
        rows = []
        for t in range(8):
            for _ in range(int(rng.integers(1, 3))):
                m = int(rng.integers(1, 33)); om = int(rng.integers(0, 64)); nn = int(rng.integers(1, 6))
                on = int(rng.integers(0, 8)); mode = [S.R, S.W, S.RW][int(rng.integers(0, 3))]
                rows.append((t, S.MATRIX, mode, int(rng.random() < 0.2), 4096 + 8 * 24, 64, om, on, m, nn, 8))
        yield f"plan_mat_wrap_{seed}", np.array(rows, dtype=S.REC)
    for seed in range(3):
        rng = np.random.default_rng(seed)
        rows = []
        for t in range(8):
            for _ in range(int(rng.integers(1, 3))):
                a = 4096 + int(rng.integers(0, 512)) * 8
                b = a + int(rng.integers(1, 64)) * 8
                rows.append((t, S.SEGMENT, [S.R, S.W, S.RW][int(rng.integers(0, 3))], int(rng.random() < 0.2), a, b, 0, 0, 0, 0, 0))
        yield f"plan_seg_{seed}", np.array(rows, dtype=S.REC)


def ref_plan_registered(recs, events):
    """ref_plan with registration events (int64 rows {before_task, kind 1 register / 2 unregister,
    ptr, size}): the reference's trees split at the registered pages."""
    with tempfile.TemporaryDirectory() as d:
        p, e = os.path.join(d, "s.bin"), os.path.join(d, "e.bin")
        S.write_stream(p, recs)
        np.asarray(events, dtype="<i8").reshape(-1, 4).tofile(e)
        subprocess.run([os.path.join(REPO, "oracle/_ref/ref_plan"), p, os.path.join(d, "o"), e],
                       check=True, capture_output=True)
        plan = np.fromfile(os.path.join(d, "o.plan"), dtype="<i8").reshape(-1, 14)
        allocs = np.fromfile(os.path.join(d, "o.allocs"), dtype="<i8")
        views = np.fromfile(os.path.join(d, "o.views"), dtype="<i8").reshape(-1, 5)
    if len(plan):
        plan = plan[np.lexsort(tuple(plan[:, k] for k in range(13, -1, -1)))]
    return plan, allocs, views


def register_cases():
    """(name, stream, events) for the registration-overflow fixtures: grids registered whole,
    unaligned, in two overlapping pieces, between tasks and unregistered; ld 200 (1600-byte
    columns) puts page boundaries inside columns; a segment stream; write-backs."""
    REG, UNREG = 1, 2
    n = 256 * 256 * 8
    heat = S.heat_stream(256, 256, 64, 64, 4, base_src=1 << 20, base_dst=1 << 21)
    yield "reg_heat_256_both", heat, [(0, REG, 1 << 20, n), (0, REG, 1 << 21, n)]
    una = S.heat_stream(256, 256, 64, 64, 4, base_src=(1 << 20) + 1024, base_dst=(1 << 22) + 512)
    yield "reg_heat_256_unaligned", una, [(0, REG, (1 << 20) + 1024, n), (0, REG, (1 << 22) + 512, n)]
    yield "reg_heat_256_pieces", heat, [(0, REG, 1 << 20, 300000), (0, REG, (1 << 20) + 300000, n - 300000),
                                        (0, REG, (1 << 21) + 5000, 70000)]
    m = 200 * 160 * 8
    ld200 = S.heat_stream(200, 160, 48, 48, 5, base_src=1 << 20, base_dst=(1 << 20) + m + 100)
    yield "reg_heat_ld200_midstream", ld200, [(3, REG, (1 << 20) + 777, 90000), (20, REG, (1 << 20) + m + 100, m),
                                              (41, UNREG, (1 << 20) + 777, 90000), (60, REG, (1 << 20) + 20000, 9000)]
    rng = np.random.default_rng(5)
    rows = []
    for t in range(24):
        for _ in range(int(rng.integers(1, 3))):
            a = (1 << 16) + int(rng.integers(0, 4096)) * 8
            b = a + int(rng.integers(1, 2048)) * 8
            rows.append((t, S.SEGMENT, [S.R, S.W, S.RW][int(rng.integers(0, 3))], int(rng.random() < 0.2), a, b, 0, 0, 0, 0, 0))
    yield "reg_seg", np.array(rows, dtype=S.REC), [(0, REG, (1 << 16) + 10000, 12000), (9, REG, (1 << 16) + 30000, 5000),
                                                   (15, UNREG, (1 << 16) + 10000, 100)]
    wb = S.microbench_stream(20, 3, n=256, ld=256, align=16, max_side_units=6)
    wb["reserved"] = (np.random.default_rng(1003).random(len(wb)) < 0.25).astype(np.uint16)
    yield "reg_mat_wb", wb, [(0, REG, (1 << 30) + 12345, 200000), (10, REG, (1 << 30) + 300000, 100000)]


AXPBY_CASES = [  # name, n, passes, seed, cmin bytes, cmax bytes
    ("axpby_20000_p3", 20000, 3, 11, 512, 65536),
    ("axpby_12345_p5", 12345, 5, 29, 64, 16384),
]


def ref_axpby(n, passes, seed, cmin, cmax):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "y.bin")
        env = dict(os.environ, DRIVERS="host,2", XKRT_DRIVERS="host,2")
        r = subprocess.run([os.path.join(REPO, "oracle/_ref/ref_axpby"), str(n), str(passes), str(seed), str(cmin), str(cmax), out],
                           check=True, capture_output=True, text=True, env=env, cwd=d)
        import json
        return np.fromfile(out), json.loads(r.stdout.strip().splitlines()[-1])["tasks"]


WRAP_SEEDS = (0, 14, 17, 21, 25, 43, 54, 171, 1, 2)      # the first eight diverge, the last two agree


def pointwise_edges(recs):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.bin")
        S.write_stream(p, recs)
        subprocess.run([os.path.join(REPO, "oracle/_bin/deps_oracle"), p, os.path.join(d, "o")],
                       check=True, capture_output=True)
        return S.read_edges(os.path.join(d, "o.edges"))


def main():
    which = set(sys.argv[1:]) or {"deps", "plan", "axpby", "wrap", "register"}
    if "register" in which:
        out = {}
        for name, recs, events in register_cases():
            plan, allocs, views = ref_plan_registered(recs, events)
            out[name + "__stream"] = recs
            out[name + "__events"] = np.asarray(events, dtype=np.int64).reshape(-1, 4)
            out[name + "__plan"] = plan
            out[name + "__allocs"] = allocs
            out[name + "__views"] = views
            out[name + "__plan_noreg"] = ref_plan(recs)[0]
            print(f"{name}: {len(recs)} accesses, {len(events)} events, {len(plan)} copies "
                  f"({len(out[name + '__plan_noreg'])} without them), {len(allocs)} allocations")
        np.savez_compressed(os.path.join(HERE, "register_golden.npz"), **out)
    if "wrap" in which:
        out = {}
        for seed in WRAP_SEEDS:
            recs = S.mixed_stream(40, seed)
            name = f"wrap_{seed}"
            out[name + "__stream"] = recs
            out[name + "__ref_edges"] = ref_edges(recs)
            out[name + "__pointwise_edges"] = pointwise_edges(recs)
            print(f"{name}: {len(out[name + '__ref_edges'])} reference edges, {len(out[name + '__pointwise_edges'])} point-wise")
        np.savez_compressed(os.path.join(HERE, "wrap_golden.npz"), **out)
    if "axpby" in which:
        out = {}
        for name, n, passes, seed, cmin, cmax in AXPBY_CASES:
            y, tasks = ref_axpby(n, passes, seed, cmin, cmax)
            out[name + "__params"] = np.array([n, passes, seed, cmin, cmax], dtype=np.int64)
            out[name + "__y"] = y
            out[name + "__tasks"] = np.array([tasks], dtype=np.int64)
            print(f"{name}: {tasks} tasks")
        np.savez_compressed(os.path.join(HERE, "axpby_golden.npz"), **out)
    if "deps" not in which and "plan" not in which:
        return
    out = {}
    for name, recs in cases():
        e = ref_edges(recs)
        out[name + "__stream"] = recs
        out[name + "__edges"] = e
        print(f"{name}: {len(recs)} accesses, {len(e)} unique edges")
    if "deps" in which:
        np.savez_compressed(os.path.join(HERE, "deps_golden.npz"), **out)
    if "plan" not in which:
        return
    out = {}
    for name, recs in plan_cases():
        plan, allocs, views = ref_plan(recs)
        out[name + "__stream"] = recs
        out[name + "__plan"] = plan
        out[name + "__allocs"] = allocs
        out[name + "__views"] = views
        print(f"{name}: {len(recs)} accesses, {len(plan)} copies, {len(allocs)} allocations")
    np.savez_compressed(os.path.join(HERE, "plan_golden.npz"), **out)


if __name__ == "__main__":
    main()
