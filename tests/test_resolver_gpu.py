"""GPU dependency resolver: bit-exact unique edge sets against the reference's own trees
(golden fixtures) and against the oracle restatement on larger seeded streams."""
import os

import numpy as np
import pytest

import deps_util as U
import streams as S
import xkaapi_b200 as xk

pytestmark = pytest.mark.gpu
GOLDEN = np.load(U.os.path.join(U.REPO, "tests", "golden", "deps_golden.npz"))
CASES = sorted(k[:-len("__stream")] for k in GOLDEN.files if k.endswith("__stream"))


def gpu_edges(recs, batches=1, seed=0):
    r = xk.Resolver()
    for b in (U.split_batches(recs, batches, seed) if batches > 1 else [recs]):
        if len(b):
            r.add(b)
    e = r.edges()
    r.close()
    return e


def expanded(recs):
    """Concurrent-mode handle accesses go through the handle map's expansion first."""
    if not ((recs["reserved"] >> 8) == 4).any():
        return recs
    m = xk.HandleMap()
    out = m.expand(recs)
    m.close()
    return out


@pytest.mark.parametrize("case", CASES)
def test_golden_reference_edges(torch_cuda, case):
    np.testing.assert_array_equal(gpu_edges(expanded(GOLDEN[case + "__stream"])), GOLDEN[case + "__edges"])


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("batches", [1, 5])
def test_concurrent_handle_streams_vs_oracle(torch_cuda, seed, batches):
    """Longer concurrent-mode handle streams: the GPU resolver on the expanded stream (in batches)
    against the oracle's restatement of the handle map on the stream as spawned."""
    recs = S.handle_concurrent_stream(seed + 300, n=3000)
    np.testing.assert_array_equal(gpu_edges(expanded(recs), batches, seed=seed), U.oracle_edges(recs))


@pytest.mark.parametrize("case", ["heat_1024_t128_s3", "microbench_1024_2000", "mixed_segmat_0", "mixed_mat_1"])
@pytest.mark.parametrize("batches", [2, 7])
def test_incremental_batches_equal_one_shot(torch_cuda, case, batches):
    np.testing.assert_array_equal(gpu_edges(GOLDEN[case + "__stream"], batches, seed=batches),
                                  GOLDEN[case + "__edges"])


@pytest.mark.parametrize("seed", range(4))
def test_mixed_streams_vs_oracle(torch_cuda, seed):
    recs = S.mixed_stream(300, seed + 100)
    # the oracle and the GPU agree on every stream (the reference itself diverges where matrix
    # tiles wrap the leading dimension; tests/golden/wrap_golden.npz pins that difference)
    np.testing.assert_array_equal(gpu_edges(recs), U.oracle_edges(recs))


_WRAP = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wrap_golden.npz"))


@pytest.mark.parametrize("case", sorted(k[:-len("__stream")] for k in _WRAP.files if k.endswith("__stream")))
def test_wrapped_tiles_gpu_edges_are_the_pinned_pointwise_set(torch_cuda, case):
    """On streams with tiles that wrap the leading dimension the GPU resolver gives exactly the
    point-wise edge set the fixture records beside the reference's (their difference is pinned
    by tests/test_oracle.py)."""
    np.testing.assert_array_equal(gpu_edges(_WRAP[case + "__stream"]), _WRAP[case + "__pointwise_edges"])


def test_microbench_16k_vs_oracle(torch_cuda):
    recs = S.microbench_stream(16384, 12345)
    np.testing.assert_array_equal(gpu_edges(recs, batches=3), U.oracle_edges(recs))


def test_heat_graph_100_steps_vs_oracle(torch_cuda):
    recs = S.heat_stream(1024, 1024, 128, 128, 100)
    np.testing.assert_array_equal(gpu_edges(recs, batches=5), U.oracle_edges(recs))


@pytest.mark.parametrize("which", ["microbench_32k", "heat_4096_t64_s10"])
def test_large_matrix_batches_vs_oracle(torch_cuda, which):
    # a small first batch creates the domain; the large second batch (tens of thousands of
    # matrix records on existing domains) is split over host threads when building ops
    recs = S.microbench_stream(32768, 777) if which == "microbench_32k" else S.heat_stream(4096, 4096, 64, 64, 10)
    cut = int(np.searchsorted(recs["task"], 500))
    r = xk.Resolver()
    r.add(recs[:cut]); r.add(recs[cut:])
    e = r.edges()
    r.close()
    np.testing.assert_array_equal(e, U.oracle_edges(recs))


def test_many_readers(torch_cuda):
    # 150 readers of the same rows, then a writer: the writer depends on all 150 readers
    tasks = [[("m", S.W, 1 << 20, 256, 0, 0, 64, 8, 8)]]
    tasks += [[("m", S.R, 1 << 20, 256, 0, 0, 64, 8, 8)] for _ in range(150)]
    tasks += [[("m", S.W, 1 << 20, 256, 16, 2, 8, 2, 8)]]
    recs = S.from_tuples(tasks)
    e = gpu_edges(recs)
    np.testing.assert_array_equal(e, U.oracle_edges(recs))
    assert sum(1 for p, s in e if s == 151) == 150


@pytest.mark.parametrize("nreaders,batches", [(5000, 1), (3000, 9)])
def test_thousands_of_readers_spill(torch_cuda, nreaders, batches):
    # far more readers of one region than a cell keeps inline (they spill to chained chunks,
    # across batches too); then two writers, each over part of it, depend on every reader
    tasks = [[("m", S.W, 1 << 20, 256, 0, 0, 64, 8, 8)]]
    tasks += [[("m", S.R, 1 << 20, 256, 0, 0, 64, 8, 8)] for _ in range(nreaders)]
    tasks += [[("m", S.W, 1 << 20, 256, 16, 2, 8, 2, 8)], [("m", S.W, 1 << 20, 256, 40, 5, 4, 1, 8)]]
    recs = S.from_tuples(tasks)
    e = gpu_edges(recs, batches, seed=3)
    np.testing.assert_array_equal(e, U.oracle_edges(recs))
    assert sum(1 for p, s in e if s == nreaders + 1) == nreaders


def test_spilled_readers_survive_refinement(torch_cuda):
    # readers spill in a first batch; the second batch brings new boundaries that split the
    # cells (each piece copies the spilled readers), appends readers to some pieces, and then
    # writes each piece separately
    ld, base = 512, 1 << 22
    first = [[("m", S.W, base, ld, 0, 0, 256, 16, 8)]]
    first += [[("m", S.R, base, ld, 0, 0, 256, 16, 8)] for _ in range(200)]
    second = [[("m", S.R, base, ld, 64, 4, 32, 4, 8)] for _ in range(40)]
    second += [[("m", S.W, base, ld, x, y, 16, 3, 8)] for x in (0, 60, 100, 200) for y in (0, 5, 12)]
    recs = S.from_tuples(first + second)
    cut = int(np.searchsorted(recs["task"], len(first)))
    r = xk.Resolver()
    r.add(recs[:cut]); r.add(recs[cut:])
    e = r.edges()
    r.close()
    np.testing.assert_array_equal(e, U.oracle_edges(recs))


class _DevView:
    """Wraps a raw device pointer for torch.as_tensor (CUDA array interface)."""
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def test_graph_csr_consistent(torch_cuda):
    torch = torch_cuda
    recs = S.microbench_stream(3000, 5, n=2048, ld=2048)
    r = xk.Resolver()
    r.add(recs)
    g = r.graph()
    nt, ne = g.ntasks, g.nedges
    ptr = torch.as_tensor(_DevView(g.succ_ptr, nt + 1), device="cuda").cpu().numpy()
    succ = torch.as_tensor(_DevView(g.succ, ne), device="cuda").cpu().numpy()
    npred = torch.as_tensor(_DevView(g.npred, nt), device="cuda").cpu().numpy()
    e = U.oracle_edges(recs)
    assert ne == len(e) and ptr[-1] == ne and ptr[0] == 0
    np.testing.assert_array_equal(np.diff(ptr), np.bincount(e[:, 0], minlength=nt))
    np.testing.assert_array_equal(npred, np.bincount(e[:, 1], minlength=nt))
    pairs = np.stack([np.repeat(np.arange(nt), np.diff(ptr)), succ], axis=1)
    np.testing.assert_array_equal(pairs, e)
    r.close()


def test_rejects_bad_streams(torch_cuda):
    r = xk.Resolver()
    bad = S.from_tuples([[("m", S.R, 4096, 64, 0, 0, 8, 8, 8)], [("m", S.W, 4096, 64, 0, 0, 8, 8, 8)]])
    bad["task"][1] = 5                       # task ids must be dense
    with pytest.raises(xk.XkbError):
        r.add(bad)
    bad2 = S.from_tuples([[("m", 0, 4096, 64, 0, 0, 8, 8, 8)]])    # mode 0
    with pytest.raises(xk.XkbError):
        r.add(bad2)
    bad3 = S.from_tuples([[("h", S.W, 4096)]])
    bad3["reserved"] = 4 << 8                # a concurrent access that was not expanded
    with pytest.raises(xk.XkbError) as ei:
        r.add(bad3)
    assert "xkb_handle_map_expand" in str(ei.value)
    ok = S.from_tuples([[("m", S.W, 4096, 64, 0, 0, 8, 8, 8)], [("m", S.R, 4096, 64, 0, 0, 8, 8, 8)]])
    r.add(ok)
    np.testing.assert_array_equal(r.edges(), [[0, 1]])
    r.close()


def _readers_stream(nreaders):
    tasks = [[("m", S.W, 1 << 20, 256, 0, 0, 64, 8, 8)]]
    tasks += [[("m", S.R, 1 << 20, 256, 0, 0, 64, 8, 8)] for _ in range(nreaders)]
    tasks += [[("m", S.W, 1 << 20, 256, 16, 2, 8, 2, 8)], [("m", S.W, 1 << 20, 256, 40, 5, 4, 1, 8)]]
    tasks += [[("m", S.R, 1 << 20, 256, 0, 0, 64, 8, 8)] for _ in range(nreaders // 2)]
    tasks += [[("m", S.RW, 1 << 20, 256, 0, 0, 64, 8, 8)]]
    return S.from_tuples(tasks)


@pytest.mark.parametrize("nseg,global_bins", [(2, False), (3, True), (8, False), (1, True)])
def test_time_split_resolution_same_edges(torch_cuda, monkeypatch, nseg, global_bins):
    """Every region's op list cut into nseg segments (XKB_RESOLVE_SEGMENTS forces the time-split
    kernels: one pass of PUT ops writing the state at each cut, then one CTA per region and
    segment emitting its LINK ops' edges): the reference's golden edges, the oracle's edges on
    seeded streams and in several batches, and reader lists past the inline ones (spilled before a
    cut, across cuts, added inside a segment, over several batches) give the same edge sets; with
    the global-atomic binning too (what domains of more than 12,288 regions use)."""
    monkeypatch.setenv("XKB_RESOLVE_SEGMENTS", str(nseg))
    if global_bins:                     # the binning without block-local counts (domains of many regions)
        monkeypatch.setenv("XKB_RESOLVE_BIN_GLOBAL", "1")
    for case in CASES:
        np.testing.assert_array_equal(gpu_edges(expanded(GOLDEN[case + "__stream"])), GOLDEN[case + "__edges"], err_msg=case)
    for case in ("heat_1024_t128_s3", "microbench_1024_2000", "mixed_segmat_0"):
        np.testing.assert_array_equal(gpu_edges(GOLDEN[case + "__stream"], 3, seed=nseg), GOLDEN[case + "__edges"], err_msg=case)
    for seed in range(2):
        recs = S.mixed_stream(300, seed + 100)
        np.testing.assert_array_equal(gpu_edges(recs), U.oracle_edges(recs))
    recs = S.microbench_stream(16384, 12345)
    np.testing.assert_array_equal(gpu_edges(recs), U.oracle_edges(recs))
    for nreaders, batches in ((100, 1), (3000, 1), (3000, 4)):
        recs = _readers_stream(nreaders)
        np.testing.assert_array_equal(gpu_edges(recs, batches, seed=7), U.oracle_edges(recs), err_msg=f"{nreaders} readers")
