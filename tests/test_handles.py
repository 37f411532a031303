"""Concurrent-mode handle accesses (CPU): the oracle's restatement of the reference's handle map
against the reference's own edges, and the library's stream expansion (xkb_handle_map_expand:
extra writer tasks inserted, concurrent writes resolved as reads) checked by running the oracle
on the expanded stream, which must give the reference's edges again."""
import os
import subprocess

import numpy as np
import pytest

import streams as S
import xkaapi_b200 as xk

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = np.load(os.path.join(REPO, "tests", "golden", "deps_golden.npz"))
CASES = sorted(k[:-len("__stream")] for k in GOLDEN.files if k.endswith("__stream"))
CONCURRENT = [c for c in CASES if c.startswith("handle_concurrent")]


def oracle(recs, tmp_path):
    p = str(tmp_path / "s.bin")
    S.write_stream(p, recs)
    subprocess.run([os.path.join(REPO, "oracle", "_bin", "deps_oracle"), p, str(tmp_path / "o")],
                   check=True, capture_output=True)
    return S.read_edges(str(tmp_path / "o.edges"))


def expand(recs, batches=1):
    m = xk.HandleMap()
    tasks = np.unique(recs["task"])
    cuts = [int(np.searchsorted(recs["task"], tasks[len(tasks) * k // batches])) for k in range(1, batches)]
    parts = [m.expand(b) for b in np.split(recs, cuts)]
    m.close()
    return np.concatenate(parts)


def hrec(task, mode, conc, h=0x5000):
    return (task, S.HANDLE, mode, conc << 8, h, 0, 0, 0, 0, 0, 0)


def test_concurrent_cases_present():
    assert len(CONCURRENT) >= 5


@pytest.mark.parametrize("case", CASES)
def test_expand_is_identity_without_concurrent_accesses(case):
    recs = GOLDEN[case + "__stream"]
    if ((recs["reserved"] >> 8) == 4).any():
        pytest.skip("holds concurrent accesses")
    out = expand(recs)
    ref = recs.copy()
    ref["reserved"] &= 0xFF
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("case", CONCURRENT)
@pytest.mark.parametrize("batches", [1, 3])
def test_expanded_stream_gives_reference_edges(case, batches, tmp_path):
    recs = GOLDEN[case + "__stream"]
    out = expand(recs, batches)
    assert not ((out["reserved"] >> 8) == 4).any()
    ntasks = int(out["task"].max()) + 1
    assert ntasks > int(recs["task"].max()) + 1                      # extra tasks were inserted
    assert np.all(np.diff(out["task"].astype(np.int64)) >= 0) and set(np.unique(out["task"])) == set(range(ntasks))
    np.testing.assert_array_equal(oracle(out, tmp_path), GOLDEN[case + "__edges"])


def test_diagram_edges():
    # dependency-map.hpp:200-223 and :247-262 -- ids after renumbering: T0=0, T1..T4=1..4, extra 5,
    # T5..T7=6..8, extra 9, T8, T9=10, 11, T10=12
    e = set(map(tuple, GOLDEN["handle_concurrent_diagrams__edges"].tolist()))
    want = {(0, w) for w in range(1, 5)} | {(w, 5) for w in range(1, 5)} | {(5, r) for r in (6, 7, 8)}
    want |= {(r, 9) for r in (6, 7, 8)} | {(9, 10), (9, 11), (10, 12), (11, 12)}
    assert e == want


def test_concurrent_writers_share_one_predecessor(tmp_path):
    recs = np.array([hrec(0, S.W, 1)] + [hrec(t, S.W, 4) for t in range(1, 6)] + [hrec(6, S.RW, 1)], dtype=S.REC)
    e = oracle(expand(recs), tmp_path).tolist()
    assert e == [[0, t] for t in range(1, 6)] + [[t, 6] for t in range(1, 6)]   # no extra task: no reads


def test_refused_forms():
    # a concurrent read with concurrent writes of earlier tasks pending
    bad = np.array([hrec(0, S.W, 4), hrec(1, S.R, 4)], dtype=S.REC)
    with pytest.raises(xk.XkbError) as ei:
        expand(bad)
    assert ei.value.code == xk.XKB_EINVAL and "concurrent read" in str(ei.value)
    # a task listing the handle again after an access that needs an extra writer
    bad = np.array([hrec(0, S.R, 1), hrec(1, S.R, 1), hrec(1, S.W, 4)], dtype=S.REC)
    with pytest.raises(xk.XkbError) as ei:
        expand(bad)
    assert "twice" in str(ei.value)
    # concurrent mode on a segment
    seg = np.array([(0, S.SEGMENT, S.W, 4 << 8, 64, 128, 0, 0, 0, 0, 0)], dtype=S.REC)
    with pytest.raises(xk.XkbError):
        expand(seg)


def test_refused_task_leaves_map_unchanged(tmp_path):
    m = xk.HandleMap()
    first = m.expand(np.array([hrec(0, S.R, 1), hrec(1, S.R, 1)], dtype=S.REC))
    with pytest.raises(xk.XkbError):
        m.expand(np.array([hrec(2, S.R, 1), hrec(2, S.W, 4)], dtype=S.REC))
    # the map still holds two pending reads: the next concurrent write gets an extra writer first
    rest = m.expand(np.array([hrec(2, S.W, 4)], dtype=S.REC))
    m.close()
    assert len(rest) == 2 and rest[0]["mode"] == 6 and rest[0]["task"] == 2 and rest[1]["task"] == 3
    assert rest[1]["mode"] == S.R                                     # a concurrent write resolves as a read
    e = oracle(np.concatenate([first, rest]), tmp_path).tolist()
    assert e == [[0, 2], [1, 2], [2, 3]]


def test_capacity_is_checked():
    recs = np.array([hrec(0, S.R, 1), hrec(1, S.W, 4)], dtype=S.REC)
    m = xk.HandleMap()
    out = np.zeros(2, dtype=S.REC)                                   # needs 3
    n = xk.ctypes.c_size_t()
    rc = xk.lib().xkb_handle_map_expand(m._h, recs.ctypes.data, len(recs), out.ctypes.data, len(out), xk.ctypes.byref(n))
    m.close()
    assert rc == xk.XKB_ERANGE
