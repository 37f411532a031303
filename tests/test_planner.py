"""Transfer planner (host code, no GPU): bit-exact against the reference's own memory tree
(golden plans from tests/golden/make_golden.py) -- allocation sizes and order, every copy
(kind, source and destination allocation/offset/ld, shape) and every access's device view."""
import os

import numpy as np
import pytest

import xkaapi_b200 as xk

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(REPO, "tests", "golden", "plan_golden.npz"))
CASES = sorted(k[:-len("__stream")] for k in G.files if k.endswith("__stream"))


def plan_of(recs):
    P = xk.Planner()
    views = []
    first = 0
    for i in range(len(recs)):
        if i == 0 or recs[i]["task"] != recs[i - 1]["task"]:
            first = i
        views.append(P.fetch(recs[i], i - first, 0 if recs[i]["reserved"] & 1 else 1))
    q = P.copies()
    if len(q):
        q = q[np.lexsort(tuple(q[:, k] for k in range(13, -1, -1)))]
    return q, P.allocations(), np.array(views)


@pytest.mark.parametrize("case", CASES)
def test_plan_matches_reference(case):
    recs = G[case + "__stream"]
    q, allocs, views = plan_of(recs)
    np.testing.assert_array_equal(q, G[case + "__plan"])
    np.testing.assert_array_equal(allocs.astype(np.int64), G[case + "__allocs"])
    dev = (recs["reserved"] & 1) == 0
    np.testing.assert_array_equal(views[dev], G[case + "__views"][dev][:, 2:])


def test_heat_plan_counts_per_step():
    """1024^2 FP64, 128^2 tiles: step 0 allocates 128 buffers and issues 127 H2D + 427 D2D copies;
    step 1 issues 60 H2D + 1184 D2D; from step 2 the pattern alternates 812 / 1296 D2D."""
    recs = G["plan_heat_1024_t128_s4__stream"]
    q, allocs, _ = plan_of(recs)
    per = []
    for s in range(4):
        sel = (q[:, 0] >= 64 * s) & (q[:, 0] < 64 * (s + 1))
        per.append((int((q[sel, 2] == 0).sum()), int((q[sel, 2] == 2).sum())))
    assert per == [(127, 427), (60, 1184), (0, 812), (0, 1296)]


def test_planner_rejects_view_overflow():
    import streams as S
    # nine differently shaped reads of one block: the 9th needs a 9th allocation view, where the
    # reference stops with a fatal error
    P = xk.Planner()
    for k in range(9):
        r = S.from_tuples([[("m", S.R, 1 << 20, 64, 0, 0, 8 + k, 4, 8)]])[0]
        if k < 8:
            P.fetch(r, 0, 1)
        else:
            with pytest.raises(xk.XkbError) as e:
                P.fetch(r, 0, 1)
            assert e.value.code == xk.XKB_ERANGE


def test_wrapped_tile_view_is_contiguous():
    import streams as S
    # an 8 x 2 tile whose rows wrap the leading dimension (ld 64, rows 60..67): one allocation of
    # 8*2*8 bytes, device view at its start with ld 8
    P = xk.Planner()
    v = P.fetch(S.from_tuples([[("m", S.RW, 4096, 64, 60, 0, 8, 2, 8)]])[0], 0, 1)
    assert list(P.allocations()) == [128] and list(v) == [0, 0, 8]
    c = P.copies()
    assert len(c) == 2 and set(c[:, 2]) == {xk.COPY_H2D}          # one H2D per rect of the tile


def test_resident_mode_moves_each_byte_once():
    """Resident layout: heat on one mirror per grid. Step 0 copies grid A in once (every cell);
    step 1 copies in only grid B's boundary ring, which no task writes; no later step copies
    anything; a host read of the final grid copies back exactly the interior the tasks wrote."""
    import streams as S
    nx, ts, steps = 256, 64, 4
    A, B = 1 << 30, 1 << 31
    recs = S.heat_stream(nx, nx, ts, ts, steps, base_src=A, base_dst=B)
    P = xk.Planner(resident=True)
    ra, rb = P.add_region(A, nx * nx * 8), P.add_region(B, nx * nx * 8)
    P.plan(recs, 1)
    c = P.copies(take=True)
    assert set(c[:, 2]) == {xk.COPY_H2D}
    cells = c[:, 11] * c[:, 12]
    assert int(cells[c[:, 8] == ra].sum()) == nx * nx               # every cell of A exactly once
    assert int(cells[c[:, 8] == rb].sum()) == 4 * nx - 4            # B's boundary ring
    assert c[c[:, 8] == rb, 0].min() >= (nx // ts) ** 2             # ... first needed at step 1
    final = A if steps % 2 == 0 else B
    P.fetch(S.from_tuples([[("m", S.R, final, nx, 0, 0, nx, nx, 8)]])[0], 0, 0)
    c = P.copies(take=True)
    assert set(c[:, 2]) == {xk.COPY_D2H}
    assert int((c[:, 11] * c[:, 12]).sum()) == (nx - 2) ** 2       # the interior the tasks wrote
    with pytest.raises(xk.XkbError):                                # outside every region
        P.fetch(S.from_tuples([[("m", S.R, 1 << 20, nx, 0, 0, 8, 8, 8)]])[0], 0, 1)


@pytest.mark.parametrize("seed", range(6))
def test_resident_mode_matches_model(seed):
    """Random accesses -- tiles of two matrices with different (ld, sizeof), tiles that wrap the
    leading dimension, segments, every mode incl. virtual ones, fetches to the GPU and to the
    host -- give the copies and views of the Python model of the resident planner, in order."""
    import numpy as np
    import streams as S
    from resident_model import ResidentModel
    rng = np.random.default_rng(seed)
    P, M = xk.Planner(resident=True), ResidentModel()
    # (base, ld, sizeof, columns); the first base is not a multiple of ld*sizeof, so tiles wrap
    mats = [((1 << 20) + 24, 64, 8, 40), ((1 << 21), 50, 4, 30)]
    seg_base, seg_len = 1 << 22, 5000
    for base, ld, s, cols in mats:
        assert P.add_region(base, ld * cols * s + 64) == M.add_region(base, ld * cols * s + 64)
    assert P.add_region(seg_base, seg_len) == M.add_region(seg_base, seg_len)
    modes = [S.R, S.W, S.RW, S.R | S.V, S.W | S.V]
    for t in range(300):
        mode = int(rng.choice(modes, p=[0.35, 0.2, 0.25, 0.1, 0.1]))
        kind = rng.integers(0, 3)
        if kind < 2:
            base, ld, s, cols = mats[kind]
            m, n = int(rng.integers(1, ld + 1)), int(rng.integers(1, 8))
            om, on = int(rng.integers(0, ld - m + 1)), int(rng.integers(0, cols - n))
            rec = S.from_tuples([[("m", mode, base, ld, om, on, m, n, s)]])[0]
        else:
            lo = int(rng.integers(0, seg_len - 1))
            hi = int(rng.integers(lo + 1, min(seg_len, lo + 700) + 1))
            rec = S.from_tuples([[("s", mode, seg_base + lo, seg_base + hi)]])[0]
        rec["task"] = t
        dev = int(rng.random() < 0.7)
        v = P.fetch(rec, t % 3, dev)
        assert tuple(v) == M.fetch(rec, t % 3, dev), t
        got = [tuple(int(x) for x in row) for row in P.copies(take=True)]
        assert got == M.take(), t


def _copied_bytes(copies):
    """Host byte intervals a list of D2H copies writes (merged)."""
    iv = []
    for c in copies:
        dst, ld, m, n, s = int(c[9]), int(c[10]), int(c[11]), int(c[12]), int(c[13])
        w = m * s
        for r in range(n):
            iv.append((dst + r * ld * s, dst + r * ld * s + w))
    iv.sort()
    out = []
    for a, b in iv:
        if out and a <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], b))
        else:
            out.append((a, b))
    return out


@pytest.mark.parametrize("seed", range(4))
def test_flush_to_host_matches_write_back_fetches(seed):
    """After random device work, flushing the resident planner copies back exactly the bytes
    that fetching every device-written record to the host copies, and leaves the host coherent
    (a second flush copies nothing)."""
    import numpy as np
    import streams as S
    rng = np.random.default_rng(100 + seed)
    mats = [((1 << 20) + 24, 64, 8, 40), ((1 << 21), 50, 4, 30)]
    seg_base, seg_len = 1 << 22, 5000
    stream = []
    for t in range(250):
        mode = int(rng.choice([S.R, S.W, S.RW]))
        kind = rng.integers(0, 3)
        if kind < 2:
            base, ld, s, cols = mats[kind]
            m, n = int(rng.integers(1, ld + 1)), int(rng.integers(1, 8))
            om, on = int(rng.integers(0, ld - m + 1)), int(rng.integers(0, cols - n))
            rec = S.from_tuples([[("m", mode, base, ld, om, on, m, n, s)]])[0]
        else:
            lo = int(rng.integers(0, seg_len - 1))
            hi = int(rng.integers(lo + 1, min(seg_len, lo + 700) + 1))
            rec = S.from_tuples([[("s", mode, seg_base + lo, seg_base + hi)]])[0]
        rec["task"] = t
        stream.append((rec, int(rng.random() < 0.8)))

    def replay():
        P = xk.Planner(resident=True)
        for base, ld, s, cols in mats:
            P.add_region(base, ld * cols * s + 64)
        P.add_region(seg_base, seg_len)
        for rec, dev in stream:
            P.fetch(rec, 0, dev)
        P.copies(take=True)
        return P

    P1, P2 = replay(), replay()
    for rec, dev in stream:
        if dev and rec["mode"] & S.W:
            r = rec.copy()
            r["mode"] = S.R
            P1.fetch(r, 0, 0)
    P2.flush_to_host()
    a, b = P1.copies(take=True), P2.copies(take=True)
    assert len(b) and set(b[:, 2]) == {xk.COPY_D2H}
    assert _copied_bytes(a) == _copied_bytes(b)
    P2.flush_to_host()
    assert len(P2.copies(take=True)) == 0


def _byte_set(copies, kind):
    """Host byte intervals (merged) that the copies of one kind read (H2D) or write (D2H)."""
    col = 5 if kind == xk.COPY_H2D else 9
    ldc = 6 if kind == xk.COPY_H2D else 10
    iv = []
    for c in copies[copies[:, 2] == kind]:
        base, ld, m, n, s = int(c[col]), int(c[ldc]), int(c[11]), int(c[12]), int(c[13])
        for r in range(n):
            a = base + r * ld * s if ld else base
            iv.append((a, a + m * s))
    iv.sort()
    out = []
    for a, b in iv:
        if out and a <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], b))
        else:
            out.append((a, b))
    return out


def _spans(recs):
    """Merged host byte spans the records touch (regions for the resident planner)."""
    iv = []
    for r in recs:
        if r["type"] == 1:                                          # segment [addr, ld)
            iv.append((int(r["addr"]), int(r["ld"])))
        else:
            s = int(r["sizeof_type"])
            a = int(r["addr"]) + (int(r["offset_n"]) * int(r["ld"]) + int(r["offset_m"])) * s
            iv.append((a, a + ((int(r["n"]) - 1) * int(r["ld"]) + int(r["m"])) * s))
    iv.sort()
    out = []
    for a, b in iv:
        if out and a <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], b))
        else:
            out.append((a, b))
    return out


def _minus(a, b):
    """Interval set difference a - b (both merged, sorted)."""
    out, j = [], 0
    for lo, hi in a:
        cur = lo
        while j < len(b) and b[j][1] <= cur:
            j += 1
        k = j
        while k < len(b) and b[k][0] < hi:
            if b[k][0] > cur:
                out.append((cur, b[k][0]))
            cur = max(cur, b[k][1])
            k += 1
        if cur < hi:
            out.append((cur, hi))
    return out


def _device_written(recs):
    """Merged host byte spans of the device fetches with W mode (rows of matrices, segments)."""
    iv = []
    for r in recs:
        if (r["reserved"] & 1) or not (r["mode"] & 2):
            continue
        if r["type"] == 1:
            iv.append((int(r["addr"]), int(r["ld"])))
        else:
            s, ld = int(r["sizeof_type"]), int(r["ld"])
            a = int(r["addr"]) + (int(r["offset_n"]) * ld + int(r["offset_m"])) * s
            iv += [(a + k * ld * s, a + k * ld * s + int(r["m"]) * s) for k in range(int(r["n"]))]
    iv.sort()
    out = []
    for a, b in iv:
        if out and a <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], b))
        else:
            out.append((a, b))
    return out


def _rec_bytes(r):
    """Merged host byte spans of one record."""
    if r["type"] == 1:
        return [(int(r["addr"]), int(r["ld"]))]
    s, ld = int(r["sizeof_type"]), int(r["ld"])
    a = int(r["addr"]) + (int(r["offset_n"]) * ld + int(r["offset_m"])) * s
    iv = sorted((a + k * ld * s, a + k * ld * s + int(r["m"]) * s) for k in range(int(r["n"])))
    out = []
    for lo, hi in iv:
        if out and lo <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], hi))
        else:
            out.append((lo, hi))
    return out


def _union(a, b):
    out = []
    for lo, hi in sorted(a + b):
        if out and lo <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], hi))
        else:
            out.append((lo, hi))
    return out


def _inter(a, b):
    return _minus(a, _minus(a, b))


@pytest.mark.parametrize("case", CASES)
def test_resident_copy_set_derives_from_reference_plan(case):
    """The resident mode (the C API's default layout: one mirror per registered region) moves the
    host bytes the reference's memory tree moves, on every golden stream:
    * H2D: the set of host bytes its copies read equals the set the reference's copies read (the
      reference may read a byte again into another allocation view; one mirror needs it once);
    * D2H, fetch by fetch: the bytes it copies back for a host access that reads are exactly the
      bytes of the access that a device access wrote since the host last had them (none for a host
      access that only writes) -- and the reference copies those too; what the reference copies besides is data the host already holds: bytes the GPU
      only read (its memory tree does not keep the host's bit when it copies a block to the device,
      memory-tree.hpp:1110-1215) or bytes a host access wrote since (the memory tree treats a host
      fetch as a read and leaves the device views coherent).
    The reference's D2D copies between allocation views have no counterpart: one mirror holds
    every view of a block."""
    recs = G[case + "__stream"]
    ref = G[case + "__plan"]
    P = xk.Planner(resident=True)
    for a, b in _spans(recs):
        P.add_region(a, b - a)
    for i in range(len(recs)):
        first = i if i == 0 or recs[i]["task"] != recs[i - 1]["task"] else first
        P.fetch(recs[i], i - first, 0 if recs[i]["reserved"] & 1 else 1)
    res = P.copies()
    assert not (res[:, 2] == xk.COPY_D2D).any()
    assert _byte_set(res, xk.COPY_H2D) == _byte_set(ref, xk.COPY_H2D)
    fresh = []                    # bytes whose newest data is on the GPU only
    for i in range(len(recs)):
        r = recs[i]
        first = i if i == 0 or recs[i]["task"] != recs[i - 1]["task"] else first
        span = _rec_bytes(r)
        if not r["reserved"] & 1:
            if r["mode"] & 2:
                fresh = _union(fresh, span)
            continue
        key = lambda q: q[(q[:, 0] == int(r["task"])) & (q[:, 1] == i - first)]
        mine, theirs = _byte_set(key(res), xk.COPY_D2H), _byte_set(key(ref), xk.COPY_D2H)
        assert mine == (_inter(span, fresh) if r["mode"] & 1 else []), i     # a host write needs no data
        assert _minus(mine, theirs) == [], i
        fresh = _minus(fresh, span)           # the host holds the newest data of the access now


def _run_plan_on_bytes(copies, host, base, dev, offs):
    """Execute copy records on byte arrays: `host` holds the host memory from address `base`,
    `dev` the device budget (allocation k at offs[k])."""
    for c in copies:
        kind, m, n, s = int(c[2]), int(c[11]), int(c[12]), int(c[13])
        w = m * s
        def rows(dev_side, alloc, off, ld):
            buf, b0 = (dev, int(offs[alloc]) + off) if dev_side else (host, off - base)
            pitch = ld * s if ld else w
            return [(buf, b0 + r * pitch) for r in range(n)]
        src = rows(kind != 0, int(c[4]), int(c[5]), int(c[6]))
        dst = rows(kind != 1, int(c[8]), int(c[9]), int(c[10]))
        for (sb, so), (db, do) in zip(src, dst):
            db[do:do + w] = sb[so:so + w]


@pytest.mark.parametrize("budget_mb,steps", [(12, 6), (3, 4)])
def test_budget_eviction_runs_heat_bit_exact_on_cpu(budget_mb, steps):
    """Reference mode with a device budget smaller than the two grids (2 x 8 MiB): the planner's
    allocations stay inside the budget without overlapping, evictions write dirty blocks back to
    the host, and executing its copies on byte arrays with each tile computed on its device views
    gives the oracle's grid, bit for bit."""
    import sys
    import streams as S
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import kernels_oracle as O
    n, ts = 1024, 128
    base = 1 << 30
    recs = S.heat_stream(n, n, ts, ts, steps, base_src=base, base_dst=base + n * n * 8)
    g = O.heat_init(n, n, seed=8)
    host = np.zeros(2 * n * n * 8, np.uint8)
    host[:n * n * 8] = g.view(np.uint8).ravel()
    host[n * n * 8:] = g.view(np.uint8).ravel()
    budget = budget_mb << 20
    dev = np.zeros(budget, np.uint8)
    P = xk.Planner(budget=budget)
    live = {}
    for t in range(len(recs) // 2):
        views = []
        for a in range(2):          # each fetch's copies run before the next fetch (as the runtime does)
            views.append(P.fetch(recs[2 * t + a], a, 1))
            offs, live = P.offsets()
            sizes = P.allocations()
            spans = sorted((int(offs[k]), int(offs[k]) + (int(sizes[k]) + 255) // 256 * 256) for k in range(len(offs)) if live[k])
            assert all(e <= budget for _, e in spans)
            assert all(spans[i][1] <= spans[i + 1][0] for i in range(len(spans) - 1))
            _run_plan_on_bytes(P.copies(take=True), host, base, dev, offs)
        # the tile body on the task's two device views (src: halo tile, dst: interior tile)
        r0, r1 = recs[2 * t], recs[2 * t + 1]
        (a0, o0, l0), (a1, o1, l1) = views
        src = dev[offs[a0] + o0:].view(np.float64) if (offs[a0] + o0) % 8 == 0 else None
        assert src is not None
        m0, n0 = int(r0["m"]), int(r0["n"])
        S0 = np.lib.stride_tricks.as_strided(src, shape=(n0, m0), strides=(l0 * 8, 8))
        D = O._update(S0.astype(np.float64), 0.2)         # interior of the halo tile = the W tile
        dst = dev[offs[a1] + o1:].view(np.float64)
        m1, n1 = int(r1["m"]), int(r1["n"])
        D1 = np.lib.stride_tricks.as_strided(dst, shape=(n1, m1), strides=(l1 * 8, 8))
        ox, oy = int(r1["offset_m"]) - int(r0["offset_m"]) - 1, int(r1["offset_n"]) - int(r0["offset_n"]) - 1
        D1[:, :] = D[oy:oy + n1, ox:ox + m1]
    # write-back of every written access, in spawn order
    for t in range(len(recs) // 2):
        w = recs[2 * t + 1].copy()
        w["mode"] = S.R
        P.fetch(w, 1, 0)
    _run_plan_on_bytes(P.copies(take=True), host, base, dev, P.offsets()[0])
    final = host[(steps % 2) * n * n * 8:][:n * n * 8].view(np.float64).reshape(n, n)
    np.testing.assert_array_equal(final, O.heat_run(g, n, n, steps, 0.2))
    evicted, written = P.eviction_stats()
    assert evicted > 0 and written > 0


@pytest.mark.parametrize("coherent", [False, True])
def test_reference_writeback_pick_and_the_coherent_one(coherent):
    """Executing the reference's plan for 4 heat steps (1024^2, 128^2 tiles) on byte arrays, then
    its host fetch of every written access: with the reference's pick of the source view (the
    largest allocation, memory-tree.hpp:1110-1160) 14,259 cells of the host grid are stale; with
    xkb_planner_set_writeback_coherent (what the C API's reference mode sets) the grid is the
    oracle's, bit for bit. The device-side plan is the same either way."""
    import sys
    import streams as S
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import kernels_oracle as O
    n, ts, steps, base = 1024, 128, 4, 1 << 30
    recs = S.heat_stream(n, n, ts, ts, steps, base_src=base, base_dst=base + n * n * 8)
    g = O.heat_init(n, n, seed=4)
    host = np.concatenate([g.view(np.uint8).ravel()] * 2)
    P = xk.Planner()
    if coherent:
        xk.check(xk.lib().xkb_planner_set_writeback_coherent(P._h, 1))
    dev = np.zeros(64 << 20, np.uint8)

    def offsets():
        sizes = P.allocations()
        return np.concatenate([[0], np.cumsum((sizes.astype(np.int64) + 255) // 256 * 256)])[:len(sizes)]
    for t in range(len(recs) // 2):
        views = []
        for a in range(2):
            views.append(P.fetch(recs[2 * t + a], a, 1))
            _run_plan_on_bytes(P.copies(take=True), host, base, dev, offsets())
        offs = offsets()
        r0, r1 = recs[2 * t], recs[2 * t + 1]
        (a0, o0, l0), (a1, o1, l1) = views
        S0 = np.lib.stride_tricks.as_strided(dev[offs[a0] + o0:].view(np.float64), shape=(int(r0["n"]), int(r0["m"])), strides=(l0 * 8, 8))
        D = O._update(S0.astype(np.float64), 0.2)
        D1 = np.lib.stride_tricks.as_strided(dev[offs[a1] + o1:].view(np.float64), shape=(int(r1["n"]), int(r1["m"])), strides=(l1 * 8, 8))
        ox, oy = int(r1["offset_m"]) - int(r0["offset_m"]) - 1, int(r1["offset_n"]) - int(r0["offset_n"]) - 1
        D1[:, :] = D[oy:oy + int(r1["n"]), ox:ox + int(r1["m"])]
    for t in range(len(recs) // 2):
        w = recs[2 * t + 1].copy()
        w["mode"] = S.R
        P.fetch(w, 1, 0)
    _run_plan_on_bytes(P.copies(take=True), host, base, dev, offsets())
    final = host[(steps % 2) * n * n * 8:][:n * n * 8].view(np.float64).reshape(n, n)
    stale = int((final != O.heat_run(g, n, n, steps, 0.2)).sum())
    assert stale == (0 if coherent else 14259)


@pytest.mark.parametrize("resident", [False, True])
def test_invalidate_fetches_from_the_host_again(resident):
    """After xkb_planner_invalidate (what xkrt_reset does to the coherency state, the reference's
    runtime_t::reset, src/memory/invalidate.cc:66-133) the same reads copy the same bytes from
    the host again; without it they copy nothing. Reference mode restarts its allocations."""
    import streams as S
    base = 1 << 30
    recs = S.from_tuples([[("m", S.R, base, 256, 0, 0, 64, 32, 8)], [("m", S.RW, base, 256, 64, 0, 64, 32, 8)]])
    P = xk.Planner(resident=resident)
    if resident:
        P.add_region(base, 256 * 64 * 8)
    for i, r in enumerate(recs):
        P.fetch(r, 0, 1)
    first = P.copies(take=True)
    assert len(first) and (first[:, 2] == 0).all()
    allocs0 = P.allocations()
    for r in recs:
        P.fetch(r, 0, 1)
    assert len(P.copies(take=True)) == 0             # both reads already coherent on the device
    P.invalidate()
    for r in recs:
        P.fetch(r, 0, 1)
    again = P.copies(take=True)
    np.testing.assert_array_equal(again, first)
    np.testing.assert_array_equal(P.allocations(), allocs0)


def test_invalidate_refuses_untaken_copies():
    import streams as S
    P = xk.Planner()
    P.fetch(S.from_tuples([[("m", S.R, 1 << 30, 256, 0, 0, 64, 32, 8)]])[0], 0, 1)
    with pytest.raises(xk.XkbError):
        P.invalidate()


RG = np.load(os.path.join(REPO, "tests", "golden", "register_golden.npz"))
REG_CASES = sorted(k[:-len("__stream")] for k in RG.files if k.endswith("__stream"))


@pytest.mark.parametrize("case", REG_CASES)
def test_registration_splits_match_reference(case):
    """Registration-overflow protection (the reference's default build): host ranges registered
    or unregistered before given tasks split the partition at their pages; every copy, allocation
    and device view equals the reference's memory tree fed the same events (golden from
    oracle/_ref/ref_plan), and differs from the plan without the registrations."""
    recs, events = RG[case + "__stream"], RG[case + "__events"]
    P = xk.Planner()
    views, first, e = [], 0, 0
    for i in range(len(recs)):
        if i == 0 or recs[i]["task"] != recs[i - 1]["task"]:
            first = i
            while e < len(events) and events[e][0] <= recs[i]["task"]:
                (P.register if events[e][1] == 1 else P.unregister)(int(events[e][2]), int(events[e][3]))
                e += 1
        views.append(P.fetch(recs[i], i - first, 0 if recs[i]["reserved"] & 1 else 1))
    q = P.copies()
    q = q[np.lexsort(tuple(q[:, k] for k in range(13, -1, -1)))]
    np.testing.assert_array_equal(q, RG[case + "__plan"])
    np.testing.assert_array_equal(P.allocations().astype(np.int64), RG[case + "__allocs"])
    dev = (recs["reserved"] & 1) == 0
    np.testing.assert_array_equal(np.array(views)[dev], RG[case + "__views"][dev][:, 2:])
    assert len(q) > len(RG[case + "__plan_noreg"])
    np.testing.assert_array_equal(plan_of(recs)[0], RG[case + "__plan_noreg"])


def test_registration_refused_in_resident_mode():
    P = xk.Planner(resident=True)
    with pytest.raises(xk.XkbError):
        P.register(1 << 20, 4096)


def test_replace_regions_keeps_block_states():
    """Resident mode: two regions replaced by their union (what overlapping registrations do in the
    C API): blocks made coherent on the GPU before stay coherent (no copy), new blocks copy from
    the host, and copies name the new region's ordinal and offsets in it."""
    import streams as S
    base = 1 << 30
    P = xk.Planner(resident=True)
    P.add_region(base, 4096)
    P.add_region(base + 4096, 4096)
    P.fetch(S.from_tuples([[("s", S.R, base, base + 1024)]])[0], 0, 1)
    assert len(P.copies(take=True)) == 1
    with pytest.raises(xk.XkbError):
        P.replace_regions(base + 8, 4096)                # a region would cross the range's start
    rid = P.replace_regions(base, 8192)
    assert rid == 2
    P.fetch(S.from_tuples([[("s", S.R, base, base + 1024)]])[0], 0, 1)
    assert len(P.copies(take=True)) == 0                 # still coherent on the GPU
    P.fetch(S.from_tuples([[("s", S.R, base + 4000, base + 5000)]])[0], 0, 1)
    q = P.copies(take=True)
    assert len(q) == 1 and q[0, 2] == 0 and q[0, 8] == rid and q[0, 9] == 4000 and q[0, 11] == 1000
