"""Helpers shared by dependency tests: run the oracle restatement on a stream."""
import os
import subprocess
import tempfile

import numpy as np

import streams as S

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_edges(recs):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.bin")
        S.write_stream(p, recs)
        subprocess.run([os.path.join(REPO, "oracle", "_bin", "deps_oracle"), p, os.path.join(d, "o")],
                       check=True, capture_output=True)
        return S.read_edges(os.path.join(d, "o.edges"))


def split_batches(recs, nbatches, seed=0):
    """Cut a stream at task boundaries into nbatches pieces."""
    tasks = np.unique(recs["task"])
    rng = np.random.default_rng(seed)
    cuts = np.sort(rng.choice(tasks[1:], size=min(nbatches - 1, len(tasks) - 1), replace=False)) if len(tasks) > 1 else []
    idx = [np.searchsorted(recs["task"], c) for c in cuts]
    return np.split(recs, idx)
