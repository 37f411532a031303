"""Regenerates tests/golden/deps_golden.npz from the REFERENCE's own dependency trees.

Each case is a seeded access stream (tests/streams.py) run through oracle/_ref/ref_deps,
which drives the reference's KBLASDependencyTree / IntervalDependencyTree via
src/task/task.cc:task_dependency_resolve (built by oracle/ref/build_ref.sh). The stream
records and the reference's unique (pred, succ) task pairs are stored side by side, so the
fixtures pin the oracle restatement and the GPU resolver without the reference present.

Known-answer cases restate the reference's own ordering tests:
  tests/task-dependency-interval.cc:86-121         W/R/RW chain on overlapping intervals
  tests/task-dependency-interval-matrix.cc:84-160  interval W -> matrix W -> interval W
Run: python tests/golden/make_golden.py   (needs oracle/_ref/ref_deps; see oracle/ref/build_ref.sh)
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


def cases():
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
    for kind in ("mat", "seg", "segmat"):
        for seed in range(3):
            yield f"mixed_{kind}_{seed}", mixed(kind, seed)


def main():
    out = {}
    for name, recs in cases():
        e = ref_edges(recs)
        out[name + "__stream"] = recs
        out[name + "__edges"] = e
        print(f"{name}: {len(recs)} accesses, {len(e)} unique edges")
    np.savez_compressed(os.path.join(HERE, "deps_golden.npz"), **out)


if __name__ == "__main__":
    main()
