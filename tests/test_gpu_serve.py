"""GPU: serving (dk_server_*): continuous admission with per-request k and L.

Every request must return exactly what the reference's single-query search returns (the
oracle, bit for bit: ids, distances, comparison and hop counts), whether it runs alone or in
a mix of other requests with different k and L, and exactly what the batch entry point
returns for the same query.
"""

import numpy as np
import pytest

from diskann_b200 import (ANNError, BF16, DiskANNIndex, FullPrecision, GpuProvider, Hybrid,
                          Knn, Metric, PQData, SearchServer, Status)
from oracle import oracle as O
from tests.helpers import queries_like, random_index, simple_pq

pytestmark = pytest.mark.gpu


def _collect(srv, tickets):
    return {t: srv.wait(t, k) for t, k in tickets}


def test_mixed_k_and_l_match_the_oracle():
    v, a, d, n = random_index(4000, 64, 24, seed=11)
    q = queries_like(v[:n], 120, seed=3)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    srv = SearchServer(prov, FullPrecision(), max_k=20, max_l=160, queue_depth=256)
    rng = np.random.default_rng(5)
    kl = []
    for _ in range(len(q)):
        k = int(rng.integers(1, 21))
        kl.append((k, int(rng.integers(k, 161))))
    tickets = [(srv.submit(q[i], k, l), k) for i, (k, l) in enumerate(kl)]
    got = _collect(srv, tickets)
    for i, ((t, _), (k, l)) in enumerate(zip(tickets, kl)):
        ids, dists, st = got[t]
        oi, od, os_ = orc.search(q[i : i + 1], k, l, 1, O.STRATEGY_FULL_PRECISION)
        np.testing.assert_array_equal(ids, oi[0])
        np.testing.assert_array_equal(dists.view(np.uint32), od[0].view(np.uint32))
        assert st["cmps"] == os_["cmps"][0] and st["hops"] == os_["hops"][0]
        assert st["result_count"] == os_["result_count"][0]
    assert srv.info()["launches"] >= 1
    srv.close()


def test_result_is_the_same_alone_and_in_the_mix():
    v, a, d, n = random_index(5000, 96, 32, seed=12)
    q = queries_like(v[:n], 200, seed=4)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    srv = SearchServer(prov, FullPrecision(), max_k=10, max_l=200, queue_depth=512, streams=3)
    alone = srv.wait(srv.submit(q[0], 10, 100), 10)
    rng = np.random.default_rng(9)
    tickets = []
    probe = None
    for i in range(1, len(q)):
        if i == 100:
            probe = srv.submit(q[0], 10, 100)
        tickets.append((srv.submit(q[i], 10, int(rng.integers(10, 201))), 10))
    mixed = srv.wait(probe, 10)
    _collect(srv, tickets)
    np.testing.assert_array_equal(alone[0], mixed[0])
    np.testing.assert_array_equal(alone[1].view(np.uint32), mixed[1].view(np.uint32))
    assert alone[2]["cmps"] == mixed[2]["cmps"]
    srv.close()


@pytest.mark.parametrize("strategy", ["hybrid", "bf16"])
def test_serving_matches_the_batch_entry_point(strategy):
    v, a, d, n = random_index(3000, 128, 24, seed=13)
    q = queries_like(v[:n], 64, seed=6)
    pq = None
    if strategy == "hybrid":
        off, piv, codes = simple_pq(v, 16, seed=2)
        pq = PQData(off, piv, codes)
    prov = GpuProvider(v, a, d, n, Metric.L2, pq=pq, low_precision=("bf16",))
    strat = Hybrid() if strategy == "hybrid" else BF16()
    bi, bd, bs = DiskANNIndex(prov).search(Knn(10, 64, 1), strat, q)
    srv = SearchServer(prov, strat, max_k=10, max_l=64, queue_depth=64)
    tickets = [(srv.submit(q[i], 10, 64), 10) for i in range(len(q))]
    got = _collect(srv, tickets)
    for i, (t, _) in enumerate(tickets):
        ids, dists, st = got[t]
        np.testing.assert_array_equal(ids, bi[i])
        np.testing.assert_array_equal(dists.view(np.uint32), bd[i].view(np.uint32))
        assert st["cmps"] == bs["cmps"][i]
    srv.close()


def test_spilled_requests_rerun_exactly(monkeypatch):
    monkeypatch.setenv("DK_HASH_LOG2", "6")
    monkeypatch.setenv("DK_GTABLE_LOG2", "8")
    v, a, d, n = random_index(4000, 64, 32, seed=14)
    q = queries_like(v[:n], 24, seed=8)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    ref = orc.search(q, 10, 200, 1, O.STRATEGY_FULL_PRECISION)
    srv = SearchServer(GpuProvider(v, a, d, n, Metric.L2), FullPrecision(), max_k=10,
                       max_l=200, queue_depth=32)
    tickets = [(srv.submit(q[i], 10, 200), 10) for i in range(len(q))]
    got = _collect(srv, tickets)
    spilled = 0
    for i, (t, _) in enumerate(tickets):
        ids, dists, st = got[t]
        np.testing.assert_array_equal(ids, ref[0][i])
        np.testing.assert_array_equal(dists.view(np.uint32), ref[1][i].view(np.uint32))
        assert st["cmps"] == ref[2]["cmps"][i]
        spilled += int(st["flags"]) & 1
    assert spilled > 0
    srv.close()


def test_admission_and_errors():
    v, a, d, n = random_index(2000, 64, 16, seed=15)
    q = queries_like(v[:n], 8, seed=9)
    srv = SearchServer(GpuProvider(v, a, d, n, Metric.L2), FullPrecision(), max_k=8,
                       max_l=32, queue_depth=4, streams=2)
    tickets = [srv.submit(q[i], 8, 32) for i in range(4)]
    with pytest.raises(ANNError) as e:
        srv.submit(q[4], 8, 32)
    assert e.value.status == Status.ADMISSION
    first = [srv.wait(t, 8) for t in tickets]
    with pytest.raises(ANNError) as e:
        srv.poll(tickets[0], 8)
    assert e.value.status == Status.NOT_FOUND
    again = srv.wait(srv.submit(q[0], 8, 32), 8)
    np.testing.assert_array_equal(again[0], first[0][0])
    with pytest.raises(ANNError) as e:
        srv.submit(q[0], 9, 32)
    assert e.value.status == Status.INVALID_ARGUMENT
    with pytest.raises(ANNError) as e:
        srv.submit(q[0], 8, 4)
    assert e.value.status == Status.L_LESS_THAN_K
    info = srv.info()
    assert info["slots"] > 0 and info["queue_depth"] == 4 and info["streams"] == 2
    srv.close()


def test_native_replay_matches_the_oracle_under_load():
    v, a, d, n = random_index(4000, 64, 24, seed=16)
    q = queries_like(v[:n], 200, seed=10)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    srv = SearchServer(GpuProvider(v, a, d, n, Metric.L2), FullPrecision(), max_k=20, max_l=120,
                       queue_depth=64)
    rng = np.random.default_rng(17)
    ks = rng.integers(1, 21, size=600)
    ls = np.array([int(rng.integers(k, 121)) for k in ks])
    arrivals = np.cumsum(rng.exponential(1.0 / 50000.0, size=600))  # 50k requests/s
    lat, ids, dists = srv.replay(q, ks, ls, arrivals, want_results=True)
    assert (lat > 0).all() and (lat < 10.0).all()
    for i in range(0, 600, 7):
        oi, od, _ = orc.search(q[i % 200 : i % 200 + 1], int(ks[i]), int(ls[i]), 1,
                               O.STRATEGY_FULL_PRECISION)
        np.testing.assert_array_equal(ids[i, : ks[i]], oi[0])
        np.testing.assert_array_equal(dists[i, : ks[i]].view(np.uint32), od[0].view(np.uint32))
    srv.close()


def test_replay_far_above_capacity_returns_each_request_its_own_results():
    """Every request arrives at once with a small queue depth and short and long requests in
    the same launches: requests finish and free their table slots while their launch still
    runs, and newer requests take those slots on other contexts.  Each must still get its own
    results (the reference's single-query search, bit for bit)."""
    v, a, d, n = random_index(4000, 64, 24, seed=21)
    q = queries_like(v[:n], 300, seed=22)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    srv = SearchServer(GpuProvider(v, a, d, n, Metric.L2), FullPrecision(), max_k=10,
                       max_l=300, queue_depth=16, streams=4)
    rng = np.random.default_rng(23)
    m = 3000
    ks = np.full(m, 10)
    ls = rng.choice([10, 20, 300], size=m)
    lat, ids, dists = srv.replay(q, ks, ls, np.zeros(m), want_results=True)
    srv.close()
    want = {int(l): orc.search(q, 10, int(l), 1, O.STRATEGY_FULL_PRECISION) for l in (10, 20, 300)}
    rows = np.arange(m) % q.shape[0]
    exp_ids = np.stack([want[int(ls[i])][0][rows[i]] for i in range(m)])
    exp_d = np.stack([want[int(ls[i])][1][rows[i]] for i in range(m)])
    wrong = np.flatnonzero((ids[:, :10] != exp_ids).any(1))
    assert wrong.size == 0, f"{wrong.size} of {m} requests got other results, first {wrong[:5]}"
    np.testing.assert_array_equal(dists[:, :10].view(np.uint32), exp_d.view(np.uint32))


def _oracle_check(orc, q, k, l, res):
    ids, dists, st = res
    oi, od, os_ = orc.search(q[None, :], k, l, 1, O.STRATEGY_FULL_PRECISION)
    np.testing.assert_array_equal(ids, oi[0])
    np.testing.assert_array_equal(dists.view(np.uint32), od[0].view(np.uint32))
    assert st["cmps"] == os_["cmps"][0] and st["hops"] == os_["hops"][0]


def test_cancelled_requests_and_the_server_stays_usable():
    """dk_server_cancel: a cancelled request (whether still queued or already on the device)
    polls as CANCELLED and frees its slot and memory; the others complete exactly; cancelling
    a collected ticket is NOT_FOUND; the server serves new requests afterwards."""
    v, a, d, n = random_index(20000, 64, 32, seed=21)
    q = queries_like(v[:n], 64, seed=22)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    # One launch context: while the first launch runs, later submits wait in the queue.
    srv = SearchServer(prov, FullPrecision(), max_k=10, max_l=400, queue_depth=64, streams=1)
    tickets = [srv.submit(q[i], 10, 400) for i in range(len(q))]
    cancelled = set(tickets[1::3])
    for t in cancelled:
        srv.cancel(t)
        srv.cancel(t)  # cancelling twice is harmless
    for i, t in enumerate(tickets):
        if t in cancelled:
            with pytest.raises(ANNError) as ei:
                srv.wait(t, 10)
            assert ei.value.status == Status.CANCELLED
        else:
            _oracle_check(orc, q[i], 10, 400, srv.wait(t, 10))
    with pytest.raises(ANNError) as ei:
        srv.cancel(tickets[0])
    assert ei.value.status == Status.NOT_FOUND
    assert srv.info()["reserved_bytes"] == 0
    _oracle_check(orc, q[5], 10, 100, srv.wait(srv.submit(q[5], 10, 100), 10))
    srv.close()


def test_admission_by_beam_state_memory_and_by_queue_depth():
    """A request is admitted while the device memory its beam state needs at its own L fits
    beside the outstanding requests' reservations: with a budget for a few requests, the next
    submit is rejected with ADMISSION (a host-side failure, nothing reaches the device), a
    larger L takes more of the budget, and collecting a request makes room again.  A full
    queue (queue_depth outstanding) is rejected the same way."""
    v, a, d, n = random_index(5000, 32, 24, seed=31)
    q = queries_like(v[:n], 16, seed=32)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    probe = SearchServer(prov, FullPrecision(), max_k=10, max_l=512, queue_depth=64)
    t = probe.submit(q[0], 10, 64)
    small = probe.info()["reserved_bytes"]
    probe.wait(t, 10)
    t = probe.submit(q[0], 10, 512)
    large = probe.info()["reserved_bytes"]
    probe.wait(t, 10)
    probe.close()
    assert large > 4 * small > 0
    srv = SearchServer(prov, FullPrecision(), max_k=10, max_l=512, queue_depth=64,
                       memory_bytes=3 * small + small // 2)
    held = [srv.submit(q[i], 10, 64) for i in range(3)]
    with pytest.raises(ANNError) as ei:
        srv.submit(q[3], 10, 64)
    assert ei.value.status == Status.ADMISSION and "memory" in str(ei.value)
    with pytest.raises(ANNError) as ei:
        srv.submit(q[3], 10, 512)  # never fits this budget
    assert ei.value.status == Status.ADMISSION
    _oracle_check(orc, q[0], 10, 64, srv.wait(held[0], 10))
    t = srv.submit(q[3], 10, 64)  # room again
    for i, tk in zip((1, 2, 3), held[1:] + [t]):
        _oracle_check(orc, q[i], 10, 64, srv.wait(tk, 10))
    assert srv.info()["reserved_bytes"] == 0
    srv.close()
    full = SearchServer(prov, FullPrecision(), max_k=10, max_l=64, queue_depth=2)
    t0, t1 = full.submit(q[0], 10, 64), full.submit(q[1], 10, 64)
    with pytest.raises(ANNError) as ei:
        full.submit(q[2], 10, 64)
    assert ei.value.status == Status.ADMISSION and "queue_depth" in str(ei.value)
    full.wait(t0, 10)
    full.wait(t1, 10)
    full.close()
