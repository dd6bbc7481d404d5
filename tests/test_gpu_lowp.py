"""GPU: the BF16 / FP8-E4M3 traversal strategies (no counterpart in the reference).

Traversal distances are low precision by design; the bars are:
* every returned (id, distance) carries the EXACT float32 distance of that id (the Rerank
  restated from the reference), bit for bit against the oracle's distance function;
* on a complete graph, where every point is scored, the queue holds the top-L points by the
  low-precision distance, which a plain float32 reference over the de-quantised rows (numpy)
  reproduces up to accumulation-order ties (tolerance: at most 2 boundary swaps in L);
* recall against the FP32 path stays high on a random graph.
"""

import numpy as np
import pytest

from diskann_b200 import (ANNError, BF16, FP8, DiskANNIndex, FullPrecision, GpuProvider, Knn,
                          Metric, Status)
from oracle import oracle as O
from tests.helpers import queries_like, random_index

pytestmark = pytest.mark.gpu

STRATS = {"bf16": BF16(), "fp8": FP8()}


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 -> float32 (numpy restatement)."""
    b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def fp8_e4m3_round(x: np.ndarray) -> np.ndarray:
    """Saturating round-to-nearest-even to the FP8-E4M3 grid (finite max 448)."""
    x = np.clip(x.astype(np.float64), -448.0, 448.0)
    out = np.zeros_like(x)
    nz = x != 0
    e = np.floor(np.log2(np.abs(x[nz])))
    e = np.maximum(e, -6)  # subnormal spacing below 2^-6
    step = 2.0 ** (e - 3)
    out[nz] = np.round(x[nz] / step) * step  # numpy rounds half to even
    return np.clip(out, -448.0, 448.0).astype(np.float32)


def dequantised(v: np.ndarray, kind: str) -> np.ndarray:
    if kind == "bf16":
        return bf16_round(v)
    scale = np.abs(v).max(axis=1, keepdims=True) / 448.0
    scale[scale == 0] = 1.0
    return (fp8_e4m3_round(v / scale) * scale).astype(np.float32)


@pytest.mark.parametrize("kind", ["bf16", "fp8"])
@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE_NORMALIZED,
                                    Metric.COSINE])
@pytest.mark.parametrize("dim", [64, 96, 128, 200])
def test_returned_distances_are_exact_fp32(kind, metric, dim):
    norm = metric != Metric.L2
    v, a, d, n = random_index(3000, dim, 24, seed=dim, normalize=norm, max_degree=31)
    q = queries_like(v[:n], 32, seed=7, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric, low_precision=(kind,)))
    ids, dists, st = idx.search(Knn(10, 64), STRATS[kind], q)
    assert (st["result_count"] == 10).all()
    for i in range(q.shape[0]):
        for j in range(10):
            exact = np.float32(O.distance(int(metric), q[i], v[ids[i, j]]))
            assert dists[i, j].view(np.uint32) == exact.view(np.uint32)
        assert (np.diff(dists[i]) >= 0).all()
    fi, _, _ = idx.search(Knn(10, 64), FullPrecision(), q)
    overlap = np.mean([len(set(fi[i]) & set(ids[i])) / 10 for i in range(q.shape[0])])
    # E4M3 keeps 3 mantissa bits: on unnormalised low-dimensional rows its traversal drifts
    # further from the FP32 one than BF16's (8 bits) does.
    assert overlap >= (0.9 if kind == "bf16" else 0.75), overlap


@pytest.mark.parametrize("kind", ["bf16", "fp8"])
@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT])
def test_queue_is_low_precision_top_l_on_complete_graph(kind, metric):
    rng = np.random.default_rng(3)
    n, dim, L = 300, 96, 40
    base = rng.standard_normal((n, dim)).astype(np.float32)
    if metric == Metric.INNER_PRODUCT:
        base /= np.linalg.norm(base, axis=1, keepdims=True)
    vectors = np.vstack([base, base[:1]])
    adj = np.array([[j for j in range(n + 1) if j != i][:n] for i in range(n + 1)], np.uint32)
    deg = np.full(n + 1, n, np.uint32)
    idx = DiskANNIndex(GpuProvider(vectors, adj, deg, n, metric, low_precision=(kind,)))
    q = rng.standard_normal((8, dim)).astype(np.float32)
    ids, dists, st = idx.search(Knn(L, L), STRATS[kind], q)
    deq = dequantised(vectors, kind).astype(np.float64)
    for i in range(q.shape[0]):
        if metric == Metric.L2:
            lp = ((deq[:n] - q[i].astype(np.float64)) ** 2).sum(1)
        else:
            lp = -(deq[:n] @ q[i].astype(np.float64))
        # The frozen point (a copy of row 0) takes one queue slot, so L+1 entries compete.
        top = set(np.argsort(lp, kind="stable")[:L].tolist())
        got = set(int(x) for x in ids[i])
        assert len(top & got) >= L - 3, (len(top & got), L)


def test_missing_low_precision_copy_is_an_error():
    v, a, d, n = random_index(200, 16, 8, seed=5, max_degree=8)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2, low_precision=("bf16",)))
    with pytest.raises(ANNError) as ei:
        idx.search(Knn(5, 10), FP8(), v[:2])
    assert ei.value.status == Status.NO_LOW_PRECISION
    idx.search(Knn(5, 10), BF16(), v[:2])


@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE_NORMALIZED,
                                    Metric.COSINE])
@pytest.mark.parametrize("dim", [32, 100, 128, 384])
def test_candidate_scores_of_each_strategy(metric, dim):
    """dk_score_candidates runs each strategy's traversal scorer: FullPrecision distances are
    the oracle's bit for bit; BF16 / FP8 distances equal a float64 evaluation over the stored
    (de-quantised) rows within 1e-5 of the terms' magnitude (FP32 accumulation); ids outside
    the index score NaN."""
    norm = metric != Metric.L2
    v, a, d, n = random_index(2000, dim, 16, seed=dim + 3 * int(metric), normalize=norm,
                              max_degree=20)
    q = queries_like(v[:n], 12, seed=9, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric, low_precision=("bf16", "fp8")))
    rng = np.random.default_rng(dim)
    cand = rng.integers(0, n + 1, size=(q.shape[0], 41)).astype(np.uint32)
    cand[:, -1] = n + 7
    full = idx.score(FullPrecision(), q, cand)
    assert np.isnan(full[:, -1]).all()
    for i in range(q.shape[0]):
        for j in range(40):
            exact = np.float32(O.distance(int(metric), q[i], v[cand[i, j]]))
            assert full[i, j].view(np.uint32) == exact.view(np.uint32)
    qd = q.astype(np.float64)[:, None, :]
    for kind in ("bf16", "fp8"):
        got = idx.score(STRATS[kind], q, cand)[:, :-1].astype(np.float64)
        x = dequantised(v, kind).astype(np.float64)[cand[:, :-1]]
        dot = (x * qd).sum(-1)
        mag = (np.abs(x) * np.abs(qd)).sum(-1)
        qq, xx = (qd ** 2).sum(-1), (x ** 2).sum(-1)
        if metric == Metric.L2:
            want, tol = qq + xx - 2 * dot, 1e-5 * (qq + xx + 2 * mag)
        elif metric == Metric.INNER_PRODUCT:
            want, tol = -dot, 1e-5 * mag + 1e-7
        elif metric == Metric.COSINE_NORMALIZED:
            want, tol = 1 - dot, 1e-5 * mag + 1e-6
        else:
            want = 1 - np.clip(dot / np.sqrt(qq * xx), -1, 1)
            tol = np.full(want.shape, 1e-5)
        err = np.abs(got - want)
        assert (err <= tol).all(), (kind, float((err / tol).max()))
