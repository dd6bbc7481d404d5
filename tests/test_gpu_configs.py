"""GPU parity on the benchmark's own workload shapes, not only on small random graphs.

The anchor workload (100,000 x 128 float32 from a seeded 64-component Gaussian mixture, means
U[0, 100], sigma 10, clipped to [0, 255]; Vamana R = 32, L_build = 50, alpha = 1.2, medoid start
point; 1,000 queries from the same mixture; k = 10, L = 100) is built once and searched by the
CUDA path through the C ABI and by the oracle.  Every query must give the same ids, the same
float32 distance bit patterns, the same comparison and hop counts and the same result count
(the reference's `search_internal`, diskann/src/graph/index.rs:1938-2005, with its queue,
diskann/src/neighbor/queue.rs:130-318).  The PQ-guided shape (32 x 256 codes, Hybrid: ADC
traversal and an exact FP32 rerank) is checked the same way on a 100,000-point mixture.
"""

import os
import sys

import numpy as np
import pytest

from diskann_b200 import (DiskANNIndex, FullPrecision, GpuProvider, Hybrid, Knn, Metric,
                          datasets, graph)
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu


def _assert_all_equal(gpu, orc):
    gi, gd, gs = gpu
    oi, od, os_ = orc
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))
    for f in ("cmps", "hops", "result_count"):
        np.testing.assert_array_equal(gs[f], os_[f])


@pytest.fixture(scope="module")
def anchor():
    import bench

    w = bench.WORKLOADS["fp100k"]
    base, queries = datasets.gaussian_mixture(w["n"], w["dim"], w["comps"], w["sigma"],
                                              seed=w["seed"], n_queries=w["nq"])
    vectors, adj, deg, n = graph.build_vamana(base, metric=Metric.L2, pruned_degree=w["R"],
                                              l_build=w["l_build"], alpha=w["alpha"], device=0)
    return w, vectors, adj, deg, n, queries


def test_anchor_workload_matches_oracle_for_every_query(anchor):
    w, vectors, adj, deg, n, queries = anchor
    assert queries.shape == (1000, 128) and n == 100_000
    # The start point is a copy of the medoid row (index N).
    med = graph.compute_medoid(vectors[:n])
    np.testing.assert_array_equal(vectors[n], vectors[med])
    idx = DiskANNIndex(GpuProvider(vectors, adj, deg, n, Metric.L2))
    orc = O.OracleIndex(vectors, adj, deg, n, O.METRIC_L2)
    for beam in (1, 4):
        gpu = idx.search(Knn(10, 100, beam), FullPrecision(), queries)
        ref = orc.search(queries, 10, 100, beam, O.STRATEGY_FULL_PRECISION, threads=8)
        _assert_all_equal(gpu, ref)
    assert float(gpu[2]["hops"].mean()) > 50  # a real traversal, not a few hops


def test_pq_guided_workload_matches_oracle():
    base, queries = datasets.gaussian_mixture(100_000, 128, 256, 8.0, seed=0xD15CA77 + 11,
                                              n_queries=1000)
    vectors, adj, deg, n = graph.build_vamana(base, metric=Metric.L2, pruned_degree=64,
                                              l_build=100, alpha=1.2, device=0)
    pq = graph.build_pq(vectors, 32, 100_000, seed=3)
    idx = DiskANNIndex(GpuProvider(vectors, adj, deg, n, Metric.L2, pq=pq))
    orc = O.OracleIndex(vectors, adj, deg, n, O.METRIC_L2, pq.offsets, pq.pivots, pq.codes)
    for l in (50, 200):
        gpu = idx.search(Knn(10, l), Hybrid(), queries)
        ref = orc.search(queries, 10, l, 1, O.STRATEGY_HYBRID, threads=8)
        _assert_all_equal(gpu, ref)
