"""GPU: the ground-truth helper's exact-rerank mode (a BF16 prefilter of C candidates per
query, then exact float64 distances) returns the same ids and distances as the full float64
scan (ids exactly; distances to float64 rounding), for every metric, on rows shaped like the
benchmark's large workloads."""

import numpy as np
import pytest

from diskann_b200 import datasets
from diskann_b200.groundtruth import knn_f64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("metric", [0, 1, 2, 3])
def test_prefiltered_ground_truth_equals_the_full_scan(metric):
    if metric == 2:
        base, q = datasets.gaussian_mixture(200_000, 128, 64, 8.0, seed=5, n_queries=300)
    else:
        base, q = datasets.normalized_gaussian(200_000, 384, seed=6, n_queries=300)
    ids, d = knn_f64(base, q, 10, metric, base_chunk=1 << 16)
    ids2, d2 = knn_f64(base, q, 10, metric, base_chunk=1 << 16, prefilter=256)
    np.testing.assert_array_equal(ids2, ids)
    # Both in float64; the scan expands |q|^2 - 2 q.x + |x|^2, the rerank sums (x - q)^2.
    np.testing.assert_allclose(d2, d, rtol=1e-9, atol=1e-9)
