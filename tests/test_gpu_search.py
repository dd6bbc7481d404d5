"""GPU parity: the CUDA search through the C ABI against the oracle and the golden vectors.

Bar: bit-exact ids, distances (float32 bit patterns), comparison and hop counts for the
full-precision path and the PQ paths (the kernels restate the reference's float rounding
sequence, so there is no tolerance to apply).
"""

import json
import os

import numpy as np
import pytest

from diskann_b200 import (STATS_DTYPE, ANNError, DiskANNIndex, FullPrecision, GpuProvider,
                          Hybrid, Knn, Metric, PQData, Quantized, Status, datasets)
from oracle import oracle as O
from tests.helpers import queries_like, random_index, simple_pq

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STRAT = {"full": (FullPrecision(), O.STRATEGY_FULL_PRECISION),
         "hybrid": (Hybrid(), O.STRATEGY_HYBRID),
         "quantized": (Quantized(), O.STRATEGY_QUANTIZED)}


def _grid_cases():
    with open(os.path.join(GOLDEN, "grid_search.json")) as f:
        return json.load(f)


def assert_same(gpu, orc, check_stats=True):
    gi, gd, gs = gpu
    oi, od, os_ = orc
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))
    if check_stats:
        np.testing.assert_array_equal(gs["cmps"], os_["cmps"])
        np.testing.assert_array_equal(gs["hops"], os_["hops"])
        np.testing.assert_array_equal(gs["result_count"], os_["result_count"])


@pytest.mark.parametrize("case", _grid_cases(),
                         ids=lambda c: f"d{c['grid_dims']}s{c['grid_size']}b{c['beam_width']}q{c['query'][0]:g}")
def test_grid_golden_through_abi(case):
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    ids, dists, st = idx.search(Knn(case["k"], case["l"], case["beam_width"]), FullPrecision(),
                                np.array([case["query"]], np.float32))
    assert [int(i) for i in ids[0]] == [r[0] for r in case["results"]]
    assert [float(x) for x in dists[0]] == [r[1] for r in case["results"]]
    assert int(st[0]["cmps"]) == case["comparisons"]
    assert int(st[0]["hops"]) == case["hops"]
    assert int(st[0]["result_count"]) == case["num_results"]


@pytest.fixture(params=["warp", "cta"])
def kernel(request, monkeypatch):
    """Run a test with the warp-per-query kernel and with the CTA-per-query kernel."""
    monkeypatch.setenv("DK_KERNEL", request.param)
    return request.param


@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE,
                                    Metric.COSINE_NORMALIZED])
@pytest.mark.parametrize("dim", [3, 100, 128])
@pytest.mark.parametrize("beam", [1, 4])
def test_full_precision_parity(metric, dim, beam, kernel):
    norm = metric in (Metric.COSINE_NORMALIZED, Metric.INNER_PRODUCT)
    v, a, d, n = random_index(3000, dim, 24, seed=dim + beam, normalize=norm, max_degree=31)
    q = queries_like(v[:n], 64, seed=11, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric))
    orc = O.OracleIndex(v, a, d, n, int(metric))
    for k, l in [(10, 10), (10, 64), (1, 128)]:
        gpu = idx.search(Knn(k, l, beam), FullPrecision(), q)
        assert_same(gpu, orc.search(q, k, l, beam, O.STRATEGY_FULL_PRECISION, threads=4))


@pytest.mark.parametrize("dim", [96, 384, 768])
def test_full_precision_parity_benchmark_dims(dim, kernel):
    v, a, d, n = random_index(2000, dim, 20, seed=dim, max_degree=26)
    q = queries_like(v[:n], 32, seed=5)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    gpu = idx.search(Knn(10, 100), FullPrecision(), q)
    assert_same(gpu, orc.search(q, 10, 100, 1, O.STRATEGY_FULL_PRECISION, threads=4))


@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE_NORMALIZED,
                                    Metric.COSINE])
@pytest.mark.parametrize("strategy", ["hybrid", "quantized"])
def test_pq_parity(metric, strategy, kernel):
    norm = metric != Metric.L2
    v, a, d, n = random_index(3000, 64, 24, seed=21, normalize=norm, max_degree=31)
    off, piv, codes = simple_pq(v, 16, seed=22)
    q = queries_like(v[:n], 48, seed=23, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric, pq=PQData(off, piv, codes)))
    orc = O.OracleIndex(v, a, d, n, int(metric), off, piv, codes)
    s, os_ = STRAT[strategy]
    for k, l, bw in [(10, 50, 1), (10, 100, 2), (5, 200, 1)]:
        assert_same(idx.search(Knn(k, l, bw), s, q), orc.search(q, k, l, bw, os_, threads=4))


@pytest.mark.parametrize("dim,chunks", [(100, 7), (128, 8), (96, 5)])
def test_pq_direct_cosine_parity(dim, chunks, kernel):
    """PQ traversal with the Cosine metric (DirectCosine over the pivot chunks): chunk lengths
    of 8 and more run the Strategy2x4 main loop, ragged ones the masked remainder."""
    v, a, d, n = random_index(2500, dim, 24, seed=dim + chunks, max_degree=31)
    off, piv, codes = simple_pq(v, chunks, seed=3)
    q = queries_like(v[:n], 40, seed=4)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.COSINE, pq=PQData(off, piv, codes)))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_COSINE, off, piv, codes)
    for strategy in ("quantized", "hybrid"):
        s, os_ = STRAT[strategy]
        assert_same(idx.search(Knn(10, 60, 1), s, q), orc.search(q, 10, 60, 1, os_, threads=4))


def test_spill_pass_is_exact(monkeypatch, kernel):
    """A visited set forced past its first-pass capacity runs in the bitmap spill pass with
    the same results; the warp kernel's global second level is exact as well."""
    v, a, d, n = random_index(4000, 32, 30, seed=31, max_degree=30)
    q = queries_like(v[:n], 40, seed=32)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    ref = orc.search(q, 10, 200, 1, O.STRATEGY_FULL_PRECISION, threads=4)
    # Tiny shared level: the warp kernel's visited set lives mostly in the global level.
    monkeypatch.setenv("DK_HASH_LOG2", "6")
    gpu = idx.search(Knn(10, 200), FullPrecision(), q)
    assert_same(gpu, ref)
    if kernel == "cta":
        assert (gpu[2]["flags"] & 1).all()
    # Both levels too small: every query spills.
    monkeypatch.setenv("DK_HASH_LOG2", "8")
    monkeypatch.setenv("DK_GTABLE_LOG2", "8")
    gpu = idx.search(Knn(10, 200), FullPrecision(), q)
    assert (gpu[2]["flags"] & 1).any()
    assert_same(gpu, ref)
    monkeypatch.delenv("DK_HASH_LOG2")
    monkeypatch.delenv("DK_GTABLE_LOG2")
    gpu2 = idx.search(Knn(10, 200), FullPrecision(), q)
    assert_same(gpu2, ref)


def test_multiple_frozen_points_and_duplicates(kernel):
    """Two start points; adjacency lists with repeated ids (the visited set drops repeats)."""
    v, a, d, n = random_index(1500, 16, 12, seed=41, frozen=2, max_degree=16)
    rng = np.random.default_rng(42)
    for r in rng.choice(n, 200, replace=False):
        if d[r] < 16:
            a[r, d[r]] = a[r, 0]
            d[r] += 1
    q = queries_like(v[:n], 32, seed=43)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    assert_same(idx.search(Knn(10, 40, 2), FullPrecision(), q),
                orc.search(q, 10, 40, 2, O.STRATEGY_FULL_PRECISION))


def test_nan_vectors_are_scored_not_inserted(kernel):
    v, a, d, n = random_index(800, 8, 10, seed=51, max_degree=10)
    v[::7, 3] = np.nan
    q = queries_like(np.nan_to_num(v[:n]), 16, seed=52)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    assert_same(idx.search(Knn(10, 30), FullPrecision(), q),
                orc.search(q, 10, 30, 1, O.STRATEGY_FULL_PRECISION))


@pytest.mark.parametrize("nan_every", [0, 5, 1])
def test_rerank_order_long_lists_and_nan_rows(nan_every, kernel):
    """Hybrid rerank over lists of 50-300 entries.  A coarse PQ (4 chunks) leaves the queue far
    from the exact order, so the warp kernel's top-k selection needs several sample rounds.
    Rows with a NaN coordinate reach the rerank through their finite PQ codes and sort after
    every number, in queue order (nan_every=1: nine rows in ten carry a NaN)."""
    v, a, d, n = random_index(3000, 64, 24, seed=71, max_degree=31)
    off, piv, codes = simple_pq(v, 4, seed=72)
    q = queries_like(v[:n], 32, seed=73)
    if nan_every == 5:
        v[:n:5, 7] = np.nan
    elif nan_every == 1:
        v[:n][np.arange(n) % 10 != 3, 7] = np.nan
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2, pq=PQData(off, piv, codes)))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2, off, piv, codes)
    for k, l in [(10, 50), (10, 200), (32, 300), (1, 100), (40, 120)]:
        gi, gd, gs = idx.search(Knn(k, l), Hybrid(), q)
        oi, od, os_ = orc.search(q, k, l, 1, O.STRATEGY_HYBRID, threads=4)
        np.testing.assert_array_equal(gi, oi)
        nan = np.isnan(od)
        np.testing.assert_array_equal(np.isnan(gd), nan)
        np.testing.assert_array_equal(gd[~nan].view(np.uint32), od[~nan].view(np.uint32))
        for key in ("cmps", "hops", "result_count"):
            np.testing.assert_array_equal(gs[key], os_[key])
        if nan_every == 1 and k >= 32:
            assert nan.any()


def test_k_equals_l_and_small_graph(kernel):
    v, a, d, n = random_index(50, 4, 6, seed=61, max_degree=6)
    q = queries_like(v[:n], 8, seed=62)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    for k, l in [(1, 1), (7, 7), (50, 60)]:
        assert_same(idx.search(Knn(k, l), FullPrecision(), q),
                    orc.search(q, k, l, 1, O.STRATEGY_FULL_PRECISION))


@pytest.mark.parametrize("nq", [100, 9000])
def test_device_entry_point_matches_host_entry_point(nq):
    """The host entry point returns exactly what the device entry point returns."""
    import torch

    v, a, d, n = random_index(12000, 64, 16, seed=71, max_degree=20)
    q = queries_like(v[:n], nq, seed=72)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    hi, hd, hs = idx.search(Knn(10, 50), FullPrecision(), q)
    out = (np.empty((nq, 10), np.uint32), np.empty((nq, 10), np.float32), np.empty(nq, STATS_DTYPE))
    oi, od, os_ = idx.search(Knn(10, 50), FullPrecision(), q, out=out)
    assert oi is out[0]
    np.testing.assert_array_equal(oi, hi)
    np.testing.assert_array_equal(od, hd)
    np.testing.assert_array_equal(os_, hs)
    dq = torch.from_numpy(q).cuda()
    ids = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    dists = torch.empty((nq, 10), dtype=torch.float32, device="cuda")
    st = torch.empty((nq, 4), dtype=torch.int32, device="cuda")
    idx.search_device(Knn(10, 50), FullPrecision(), dq, ids, dists, st)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ids.cpu().numpy().view(np.uint32), hi)
    np.testing.assert_array_equal(dists.cpu().numpy(), hd)
    np.testing.assert_array_equal(st.cpu().numpy()[:, 0].view(np.uint32), hs["cmps"])


def test_errors():
    v, a, d, n = random_index(100, 8, 6, seed=81, max_degree=6)
    bad = a.copy()
    bad[3, 0] = 10_000
    with pytest.raises(ANNError) as ei:
        GpuProvider(v, bad, d, n, Metric.L2)
    assert ei.value.status == Status.INVALID_GRAPH
    d2 = d.copy()
    d2[5] = 7
    with pytest.raises(ANNError) as ei:
        GpuProvider(v, a, d2, n, Metric.L2)
    assert ei.value.status == Status.INVALID_GRAPH
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    with pytest.raises(ANNError) as ei:
        idx.search(Knn(5, 10), Hybrid(), v[:2])
    assert ei.value.status == Status.NO_PQ
    with pytest.raises(ANNError) as ei:
        idx.search(Knn(5, 10), FullPrecision(), v[:2, :4])
    assert ei.value.status == Status.DIMENSION_MISMATCH
    ids, dists, st = idx.search(Knn(5, 10), FullPrecision(), np.zeros((0, 8), np.float32))
    assert ids.shape == (0, 5)
