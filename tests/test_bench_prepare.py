"""CPU: the benchmark's workload preparation — the in-memory path (no on-disk cache) with a
zero-centred mixture scaled to unit length, its float64 ground truth, and the workload
description carrying the metric."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_in_memory_normalised_mixture_workload(tmp_path, monkeypatch):
    import bench
    from diskann_b200 import datasets

    w = dict(bench.WORKLOADS["tiny"], n=1500, nq=32, normalized=True, metric=1,
             mean_range=(-50.0, 50.0), clip=(-255.0, 255.0), cache=False)
    monkeypatch.setitem(bench.WORKLOADS, "tiny_ipn", w)
    data = bench.prepare("tiny_ipn", 0, str(tmp_path))
    assert os.listdir(tmp_path) == []  # nothing written
    n = data["n"]
    assert data["vectors"].shape == (n + 1, w["dim"])
    np.testing.assert_allclose(np.linalg.norm(data["vectors"], axis=1), 1.0, rtol=1e-5)
    np.testing.assert_allclose(np.linalg.norm(data["queries"], axis=1), 1.0, rtol=1e-5)
    # Zero-centred: coordinates of both signs.
    assert (data["vectors"] < 0).mean() > 0.3
    # The same rows as the generator followed by normalize_rows.
    base, queries = datasets.gaussian_mixture(n, w["dim"], w["comps"], w["sigma"], seed=w["seed"],
                                              mean_range=w["mean_range"], clip=w["clip"],
                                              n_queries=w["nq"])
    np.testing.assert_array_equal(data["vectors"][:n], datasets.normalize_rows(base))
    np.testing.assert_array_equal(data["queries"], datasets.normalize_rows(queries))
    # Ground truth: exact top-k by inner product (largest dot first).
    dot = data["queries"].astype(np.float64) @ data["vectors"][:n].astype(np.float64).T
    want = np.argsort(-dot, axis=1, kind="stable")[:, : w["k"]]
    assert (np.sort(data["gt"], 1) == np.sort(want, 1)).mean() > 0.99
    assert data["pq"] is not None and data["pq"].codes.shape == (n + 1, w["pq_chunks"])
    cfg = bench.config_of(w, "tiny_ipn", 20, "fp32")
    assert cfg["metric"] == "INNER_PRODUCT"
    assert "means U[-50, 50]" in cfg["workload"] and "unit length" in cfg["workload"]


def test_in_memory_workload_is_single_rank(monkeypatch, tmp_path):
    import bench

    monkeypatch.setitem(bench.WORKLOADS, "tiny_mem", dict(bench.WORKLOADS["tiny"], cache=False))
    with pytest.raises(RuntimeError):
        bench.prepare("tiny_mem", 1, str(tmp_path))


def test_normalize_rows_in_place():
    from diskann_b200 import datasets

    x = np.random.default_rng(0).standard_normal((1000, 7)).astype(np.float32) * 5
    y = x.copy()
    out = datasets.normalize_rows(x, chunk=64)
    assert out is x
    np.testing.assert_allclose(x, y / np.linalg.norm(y, axis=1, keepdims=True), rtol=1e-6)
