"""CPU: the medoid start point (dk_compute_medoid, host code) against a numpy restatement of
the reference's `ComputeMedoid for f32` (diskann-utils/src/sampling/medoid.rs:15-45).

The reference sums every column in float64, divides by the row count in float64 and casts the
mean to float32; it then walks the rows in order and keeps the FIRST row whose float32
SquaredL2 to that mean is strictly smaller than the best so far (starting from f32::MAX).  The
distance is the reference's float32 SquaredL2 kernel, whose rounding order the oracle restates
(pinned elsewhere against an independent numpy restatement of the x86-64-v3 schema), so the
restatement below computes each row's distance through the oracle.
"""

import numpy as np
import pytest

from diskann_b200 import graph
from oracle import oracle as O


def _medoid_restated(data: np.ndarray) -> int:
    mean = (data.astype(np.float64).sum(axis=0) / np.float64(data.shape[0])).astype(np.float32)
    best, arg = np.float32(np.finfo(np.float32).max), None
    for i in range(data.shape[0]):
        d = np.float32(O.distance(O.METRIC_L2, mean, data[i]))
        if d < best:
            best, arg = d, i
    return arg


@pytest.mark.parametrize("seed,n,dim", [(1, 500, 3), (2, 800, 100), (3, 300, 128)])
def test_medoid_matches_restatement(seed, n, dim):
    rng = np.random.default_rng(seed)
    data = (rng.standard_normal((n, dim)) * 10 + 50).astype(np.float32)
    assert graph.compute_medoid(data) == _medoid_restated(data)


def test_medoid_first_of_tied_rows_wins():
    """Several rows at exactly the same (smallest) distance: the first one in row order."""
    rng = np.random.default_rng(7)
    data = rng.integers(0, 20, size=(400, 8)).astype(np.float32)
    mean = (data.astype(np.float64).sum(0) / 400).astype(np.float32)
    centre = np.round(mean)
    data[37] = centre
    data[120] = centre
    data[399] = centre
    got = graph.compute_medoid(data)
    assert got == _medoid_restated(data)
    assert got == 37


def test_medoid_mean_in_float64():
    """Columns whose float32 running sum loses the small parts: the float64 mean decides."""
    n = 3001
    data = np.zeros((n, 2), np.float32)
    data[:, 0] = 1.0e7
    data[::2, 1] = 1.0
    data[1::2, 1] = 2.0
    # float64 mean of column 1 is (1501 * 1 + 1500 * 2) / 3001 = 1.49983...
    data[5] = [1.0e7, 1.4998]
    data[6] = [1.0e7, 1.5003]
    assert graph.compute_medoid(data) == _medoid_restated(data) == 5
