"""CPU: the oracle's diskann-inmem search (provider.rs restated): integer distances against an
independent numpy restatement, unreadable slots visited but never scored, Translate."""

import numpy as np
import pytest

from diskann_b200.index import inmem_rows
from oracle import oracle as O
from tests.helpers import inmem_fixture


def _complete_graph(total):
    adj = np.array([[j for j in range(total) if j != i] for i in range(total)], np.uint32)
    return adj, np.full(total, total - 1, np.uint32)


def _int_distance(metric, q, x):
    """The reference's integer kernels: exact sums, one conversion to f32 (RNE), then the
    f32 post-op (simd.rs:2327-2363 for cosine)."""
    a, b = q.astype(np.int64), x.astype(np.int64)
    f = lambda v: np.float32(np.int32(np.int64(v)))  # noqa: E731
    if metric == O.METRIC_L2:
        return f(((a - b) ** 2).sum())
    if metric == O.METRIC_INNER_PRODUCT:
        return np.float32(-f((a * b).sum()))
    nx, ny, p = f((a * a).sum()), f((b * b).sum()), f((a * b).sum())
    if nx < np.finfo(np.float32).tiny or ny < np.finfo(np.float32).tiny:
        return np.float32(1.0)
    den = np.float32(np.sqrt(nx)) * np.float32(np.sqrt(ny))
    return np.float32(1.0) - np.float32(np.clip(np.float32(p / den), -1.0, 1.0))


@pytest.mark.parametrize("elem,code", [("u8", 2), ("i8", 3)])
@pytest.mark.parametrize("metric", [O.METRIC_L2, O.METRIC_INNER_PRODUCT, O.METRIC_COSINE])
def test_oracle_integer_distances(elem, code, metric):
    typed, values, _, _, n, tags, ext = inmem_fixture(elem, 40, 37, seed=3, unreadable=0.0,
                                                      unmapped=0.0)
    total = typed.shape[0]
    adj, deg = _complete_graph(total)
    ix = O.OracleIndex(values, adj, deg, n, metric)
    q = typed[5].copy()
    q[::3] = typed[9][::3]
    ids, dists, st = ix.inmem_search(code, inmem_rows(typed, tags), ext, q, n, total)
    want = {int(ext[i]): _int_distance(metric, q, typed[i]) for i in range(n)}
    assert len(ids) == n
    for i, d in zip(ids, dists):
        assert np.float32(d).view(np.uint32) == want[int(i)].view(np.uint32)
    assert (np.diff(dists) >= 0).all()


def test_oracle_unreadable_slots_are_visited_not_scored():
    typed, values, adj, deg, n, tags, ext = inmem_fixture("f32", 300, 16, seed=4,
                                                          unreadable=0.3, unmapped=0.2)
    ix = O.OracleIndex(values, adj, deg, n, O.METRIC_L2)
    ids, dists, st = ix.inmem_search(0, inmem_rows(typed, tags), ext, values[7], 20, 60)
    readable_mapped = {int(ext[i]) for i in range(n) if tags[i] >= 254 and ext[i] != 2**64 - 1}
    assert set(ids[: st["result_count"]].tolist()) <= readable_mapped
    # Everything readable: more comparisons (unreadable slots cost none).
    all_tags = np.where(np.arange(len(tags)) < n, 254, 255).astype(np.uint8)
    _, _, st_all = ix.inmem_search(0, inmem_rows(typed, all_tags), ext, values[7], 20, 60)
    assert st_all["cmps"] > st["cmps"]
