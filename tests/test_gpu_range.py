"""GPU: range search (dk_range_search, the reference's `Range`) against range_search.rs's
golden baselines and the oracle, bit for bit: result ids and distances in order, comparison
and hop counts, result count and the second-round flag."""

import json
import os

import numpy as np
import pytest

from diskann_b200 import (ANNError, DiskANNIndex, GpuProvider, KnnSearchError, Metric, Range,
                          Status, datasets)
from oracle import oracle as O
from tests.helpers import queries_like, random_index

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _cases():
    with open(os.path.join(GOLDEN, "range_search.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["source"].split("/")[-1][:-5])
def test_range_golden_through_abi(case):
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    params = Range(case["starting_l"], case["radius"], inner_radius=case["inner_radius"],
                   initial_slack=case["initial_slack"], range_slack=case["range_slack"],
                   max_returned=case["max_returned"])
    res, st = idx.range_search(params, np.array(case["query"], np.float32))
    ids, dists = res[0]
    assert [[int(i), float(x)] for i, x in zip(ids, dists)] == case["results"]
    assert int(st[0]["cmps"]) == case["comparisons"]
    assert int(st[0]["hops"]) == case["hops"]
    assert int(st[0]["result_count"]) == case["result_count"]
    assert bool(int(st[0]["flags"]) & 2) == case["second_round"]


def _assert_same(idx, orc, q, p, capacity=None):
    res, st = idx.range_search(p, q, capacity=capacity)
    for i in range(q.shape[0]):
        oi, od, os_ = orc.range_search(q[i], p.starting_l, p.radius, beam_width=p.beam_width,
                                       inner_radius=p.inner_radius, initial_slack=p.initial_slack,
                                       range_slack=p.range_slack, max_returned=p.max_returned or 0,
                                       capacity=capacity)
        np.testing.assert_array_equal(res[i][0], oi)
        np.testing.assert_array_equal(res[i][1].view(np.uint32), od.view(np.uint32))
        assert int(st[i]["cmps"]) == int(os_["cmps"]) and int(st[i]["hops"]) == int(os_["hops"])
        assert int(st[i]["flags"]) & 2 == int(os_["flags"]) & 2


@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE])
@pytest.mark.parametrize("dim", [64, 128])
def test_range_parity_with_the_oracle(metric, dim):
    norm = metric != Metric.L2
    v, a, d, n = random_index(3000, dim, 24, seed=dim + int(metric), metric=int(metric),
                              normalize=norm, max_degree=31)
    q = queries_like(v[:n], 16, seed=5, normalize=norm)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, metric))
    orc = O.OracleIndex(v, a, d, n, int(metric))
    # A radius around the 20th-nearest distance of the first query: both rounds run.
    ids0, d0, _ = orc.search(q[:1], 40, 80, 1)
    r = float(d0[0, 20])
    inner = float(d0[0, 2])
    for p in [Range(40, r), Range(40, r, inner_radius=inner), Range(40, r, beam_width=2),
              Range(40, r, range_slack=1.3, initial_slack=0.5), Range(40, r, max_returned=60),
              Range(8, r * 1.5, max_returned=120), Range(40, r, beam_width=8)]:
        _assert_same(idx, orc, q, p, capacity=p.max_returned or 4000)


def test_range_errors():
    with pytest.raises(KnnSearchError):
        Range(0, 1.0)
    with pytest.raises(ANNError):
        Range(10, 1.0, max_returned=5)
    with pytest.raises(ANNError):
        Range(10, 1.0, inner_radius=2.0)
    v, a, d, n = random_index(500, 16, 8, seed=3, max_degree=8)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    with pytest.raises(ANNError) as e:
        idx.range_search(Range(10, 1.0), v[:2, :8])
    assert e.value.status == Status.DIMENSION_MISMATCH


def test_range_device_entry_point_matches_host_entry_point():
    """dk_range_search_device (device buffers, caller's stream) returns what dk_range_search
    returns."""
    import ctypes

    import torch

    from diskann_b200 import STATS_DTYPE, _native

    v, a, d, n = random_index(3000, 64, 24, seed=77, max_degree=31)
    q = queries_like(v[:n], 40, seed=8)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    _, d0, _ = orc.search(q[:1], 40, 80, 1)
    p = Range(40, float(d0[0, 20]), max_returned=200)
    host, hst = idx.range_search(p, q, capacity=200)
    dq = torch.from_numpy(q).cuda()
    ids = torch.empty((40, 200), dtype=torch.int32, device="cuda")
    dists = torch.empty((40, 200), dtype=torch.float32, device="cuda")
    st = torch.empty((40, 4), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _native.load().dk_range_search_device(
        idx.provider.handle, dq.data_ptr(), 64, 40, p.starting_l, p.beam_width, p.radius,
        float("nan"), p.initial_slack, p.range_slack, p.max_returned, 200, ids.data_ptr(),
        dists.data_ptr(), st.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    ids_h = ids.cpu().numpy().view(np.uint32)
    d_h = dists.cpu().numpy()
    st_h = st.cpu().numpy().view(np.uint32).reshape(-1).view(STATS_DTYPE)
    for i in range(40):
        c = int(st_h[i]["result_count"])
        assert c == int(hst[i]["result_count"])
        np.testing.assert_array_equal(ids_h[i, :c], host[i][0])
        np.testing.assert_array_equal(d_h[i, :c].view(np.uint32), host[i][1].view(np.uint32))
        assert int(st_h[i]["cmps"]) == int(hst[i]["cmps"])


@pytest.mark.parametrize("capacity,radius_rank", [(40, 39), (4000, 5), (4000, 59)])
def test_host_copy_of_filled_slots_only(capacity, radius_rank):
    """The host entry point copies back only each query's filled slots (packed on the device,
    spread in place into the caller's rows) unless the rows are mostly full; either way every
    row's results equal the oracle's, also into reused caller-owned arrays.  Rows whose
    in-range set reached the capacity (flags bit 2: possibly incomplete, a bound the reference
    does not have) are not compared."""
    from diskann_b200 import STATS_DTYPE

    v, a, d, n = random_index(3000, 64, 24, seed=78, max_degree=31)
    q = queries_like(v[:n], 64, seed=9)
    idx = DiskANNIndex(GpuProvider(v, a, d, n, Metric.L2))
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    _, d0, _ = orc.search(q[:1], 60, 80, 1)
    p = Range(40, float(d0[0, radius_rank]))
    out = (np.full((64, capacity), 7, np.uint32), np.full((64, capacity), 7.0, np.float32),
           np.zeros(64, STATS_DTYPE))
    for _ in range(2):
        ids, dists, st = idx.range_search_arrays(p, q, capacity=capacity, out=out)
        assert ids is out[0] and dists is out[1] and st is out[2]
        full = (st["flags"] & 4) != 0
        assert (~full).sum() >= 16
        for i in np.flatnonzero(~full):
            oi, od, ost = orc.range_search(q[i], p.starting_l, p.radius, capacity=capacity)
            c = int(st[i]["result_count"])
            assert c == int(np.asarray(ost["result_count"]).reshape(-1)[0])
            np.testing.assert_array_equal(ids[i, :c], oi)
            np.testing.assert_array_equal(dists[i, :c].view(np.uint32), od.view(np.uint32))
