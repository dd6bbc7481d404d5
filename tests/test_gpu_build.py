"""GPU: graph construction with the batch searches on the device (dk_build_vamana_device)
produces exactly the graph of the host build (dk_build_vamana): the device searches are the
bit-exact search kernels, so every visited record, prune and back edge is the same."""

import numpy as np
import pytest

from diskann_b200 import Metric, datasets, graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("metric,dim,alpha", [(Metric.L2, 64, 1.2), (Metric.INNER_PRODUCT, 96, 1.2),
                                              (Metric.COSINE, 128, 1.2), (Metric.L2, 384, 1.2),
                                              (Metric.COSINE_NORMALIZED, 100, 1.2),
                                              (Metric.L2, 128, 1.0), (Metric.L2, 45, 1.4)])
def test_device_build_equals_host_build(metric, dim, alpha):
    """Batches of 256 or more are searched, pruned and given their back edges on the GPU."""
    if metric == Metric.L2:
        base, _ = datasets.gaussian_mixture(6000, dim, 16, 8.0, seed=dim)
    else:
        base, _ = datasets.normalized_gaussian(6000, dim, seed=dim)
    kw = dict(metric=metric, pruned_degree=24, l_build=40, alpha=alpha, max_batch=1024)
    v0, a0, d0, n0 = graph.build_vamana(base, **kw)
    v1, a1, d1, n1 = graph.build_vamana(base, device=0, **kw)
    np.testing.assert_array_equal(d0, d1)
    np.testing.assert_array_equal(a0, a1)


@pytest.mark.parametrize("env", ["DK_BUILD_POOL_CAP_FIRST", "DK_BUILD_POOL_CAP"])
def test_device_build_long_lists(monkeypatch, env):
    """Back-edge lists that outgrow the first device pool go to a second launch with a larger
    pool, and those that outgrow every pool are appended and pruned on the host."""
    monkeypatch.setenv(env, "32")
    base, _ = datasets.gaussian_mixture(4000, 64, 16, 8.0, seed=5)
    kw = dict(metric=Metric.L2, pruned_degree=24, l_build=40, alpha=1.2, max_batch=1024)
    v0, a0, d0, n0 = graph.build_vamana(base, **kw)
    v1, a1, d1, n1 = graph.build_vamana(base, device=0, **kw)
    np.testing.assert_array_equal(d0, d1)
    np.testing.assert_array_equal(a0, a1)


@pytest.mark.parametrize("metric,dim", [(Metric.L2, 128), (Metric.INNER_PRODUCT, 96)])
def test_device_build_equals_oracle_build(metric, dim):
    """The device build against the oracle's independent restatement of the construction rules
    (oracle/build.cpp): the identical graph, on enough points that most batches run on the GPU."""
    from oracle import oracle as O

    if metric == Metric.L2:
        base, _ = datasets.gaussian_mixture(20000, dim, 32, 8.0, seed=dim + 1)
    else:
        base, _ = datasets.normalized_gaussian(20000, dim, seed=dim + 1)
    kw = dict(pruned_degree=32, l_build=50, alpha=1.2, max_batch=2048)
    v0, a0, d0, n0 = graph.build_vamana(base, metric=metric, device=0, **kw)
    v1, a1, d1, n1 = O.build_vamana(base, int(metric), **kw)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(d0, d1)
    np.testing.assert_array_equal(a0, a1)
