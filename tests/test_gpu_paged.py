"""GPU: paged search (dk_paged_search_*, the reference's `PagedSearch`) against
paged_search.rs's golden pages and the oracle, bit for bit: every page's ids and distances in
order, and the sessions' running comparison and hop counts."""

import json
import os

import numpy as np
import pytest

from diskann_b200 import ANNError, DiskANNIndex, GpuProvider, Metric, Status, datasets
from oracle import oracle as O
from tests.helpers import queries_like, random_index

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _cases():
    with open(os.path.join(GOLDEN, "paged_search.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["source"].split("/")[-1][:-5])
def test_paged_golden_through_abi(case):
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    ps = idx.paged_search(np.array(case["query"], np.float32), case["search_l"])
    pages = []
    while True:
        page, _ = ps.next_page(case["page_size"])
        ids, dists = page[0]
        if len(ids) == 0:
            break
        pages.append([[int(i), float(x)] for i, x in zip(ids, dists)])
    assert pages == case["pages"]
    # Exhausted sessions stay empty.
    assert len(ps.next_page(case["page_size"])[0][0][0]) == 0
    ps.close()


def _compare(ps, ops, ks):
    for k in ks:
        pages, st = ps.next_page(k)
        for i, o in enumerate(ops):
            oi, od, os_ = o.next_page(k)
            np.testing.assert_array_equal(pages[i][0], oi)
            np.testing.assert_array_equal(pages[i][1].view(np.uint32), od.view(np.uint32))
            assert int(st[i]["cmps"]) == int(os_["cmps"]) and int(st[i]["hops"]) == int(os_["hops"])


@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE])
@pytest.mark.parametrize("dim", [64, 128])
def test_paged_parity_with_the_oracle(metric, dim):
    norm = metric != Metric.L2
    v, a, d, n = random_index(2500, dim, 24, seed=dim + int(metric), metric=int(metric),
                              normalize=norm, max_degree=31)
    q = queries_like(v[:n], 12, seed=7, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric))
    orc = O.OracleIndex(v, a, d, n, int(metric))
    for l_value, ks in [(20, [5, 3, 10, 20, 1, 7, 20, 20, 4, 13]), (50, [50, 10, 25, 50, 2, 50])]:
        ps = idx.paged_search(q, l_value)
        ops = [orc.paged_search(q[i], l_value) for i in range(len(q))]
        _compare(ps, ops, ks)
        ps.close()


def test_paged_with_init_ids_matches_the_oracle():
    v, a, d, n = random_index(3000, 96, 24, seed=21, max_degree=31)
    q = queries_like(v[:n], 8, seed=8)
    rng = np.random.default_rng(4)
    init = rng.integers(0, n, size=(len(q), 3)).astype(np.uint32)
    init[0, 1] = init[0, 0]  # a repeated init id
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    ps = idx.paged_search(q, 30, init_ids=init)
    ops = [orc.paged_search(q[i], 30, init_ids=init[i]) for i in range(len(q))]
    _compare(ps, ops, [10, 30, 5, 30, 30, 1])
    ps.close()


def test_paged_runs_to_exhaustion_without_repeats():
    v, a, d, n = random_index(400, 32, 12, seed=5, max_degree=16)
    q = queries_like(v[:n], 4, seed=3)
    ps = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2)).paged_search(q, 40)
    seen = [set() for _ in range(len(q))]
    for _ in range(40):
        pages, _ = ps.next_page(40)
        for i, (ids, dists) in enumerate(pages):
            assert not (set(ids.tolist()) & seen[i])
            assert (np.diff(dists) >= 0).all()
            assert (ids < n).all()
            seen[i].update(ids.tolist())
    assert all(len(s) > 0 for s in seen)
    ps.close()


def test_paged_errors_and_capacity():
    v, a, d, n = random_index(1000, 32, 12, seed=6, max_degree=16)
    q = queries_like(v[:n], 2, seed=2)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    ps = idx.paged_search(q, 16)
    for k in (0, 17):
        with pytest.raises(ANNError) as e:
            ps.next_page(k)
        assert e.value.status == Status.INVALID_ARGUMENT
    ps.close()
    with pytest.raises(ANNError) as e:
        idx.paged_search(q, 16, init_ids=np.full((2, 1), n + 5, np.uint32))
    assert e.value.status == Status.INVALID_ARGUMENT
    small = idx.paged_search(q, 16, queue_capacity=24)
    _, st = small.next_page(16)
    assert (st["flags"] & 4).all()
    small.close()
