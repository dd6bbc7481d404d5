"""GPU: the diskann-inmem provider (dk_inmem_*) against the oracle's restatement of its search,
bit for bit: external ids, distances, comparison and hop counts, for every element type and
metric, with unreadable slots (visited, never scored) and unmapped slots (dropped by
Translate)."""

import numpy as np
import pytest

from diskann_b200 import ANNError, InmemProvider, Knn, Metric, Status
from diskann_b200.index import inmem_rows
from oracle import oracle as O
from tests.helpers import inmem_fixture

pytestmark = pytest.mark.gpu

ELEMS = {"f32": 0, "f16": 1, "u8": 2, "i8": 3}


def _queries(typed, nq, seed):
    rng = np.random.default_rng(seed)
    src = typed[rng.choice(typed.shape[0] - 1, size=nq, replace=False)]
    if typed.dtype in (np.uint8, np.int8):
        info = np.iinfo(typed.dtype)
        noise = rng.integers(-6, 7, size=src.shape)
        return np.clip(src.astype(np.int64) + noise, info.min, info.max).astype(typed.dtype)
    return (src.astype(np.float32) + rng.standard_normal(src.shape).astype(np.float32)).astype(typed.dtype)


def _check(prov, orc, code, rows, ext, q, knn):
    ids, dists, st = prov.search(knn, q)
    for i in range(q.shape[0]):
        oq = q[i] if code >= 2 else q[i].astype(np.float32)
        oi, od, os_ = orc.inmem_search(code, rows, ext, oq, knn.k_value, knn.l_value,
                                       knn.beam_width)
        np.testing.assert_array_equal(ids[i], oi)
        np.testing.assert_array_equal(dists[i].view(np.uint32), od.view(np.uint32))
        assert int(st[i]["cmps"]) == int(os_["cmps"]) and int(st[i]["hops"]) == int(os_["hops"])
        assert int(st[i]["result_count"]) == int(os_["result_count"])


@pytest.mark.parametrize("elem", list(ELEMS))
@pytest.mark.parametrize("metric", [Metric.L2, Metric.INNER_PRODUCT, Metric.COSINE,
                                    Metric.COSINE_NORMALIZED])
@pytest.mark.parametrize("dim", [128, 45])
def test_inmem_parity_with_the_oracle(elem, metric, dim):
    typed, values, adj, deg, n, tags, ext = inmem_fixture(elem, 1500, dim, seed=dim + int(metric),
                                                          metric=int(metric))
    prov = InmemProvider(typed, adj, deg, n, tags, ext, metric)
    orc = O.OracleIndex(values, adj, deg, n, int(metric))
    rows = inmem_rows(typed, tags)
    q = _queries(typed, 10, seed=5)
    for knn in (Knn(10, 40), Knn(5, 64, 2)):
        _check(prov, orc, ELEMS[elem], rows, ext, q, knn)
    prov.close()


def test_inmem_tags_update_matches_the_oracle():
    typed, values, adj, deg, n, tags, ext = inmem_fixture("u8", 2000, 64, seed=9)
    prov = InmemProvider(typed, adj, deg, n, tags, ext, Metric.L2)
    orc = O.OracleIndex(values, adj, deg, n, O.METRIC_L2)
    q = _queries(typed, 8, seed=2)
    # Retire a block of slots, publish a few that were not readable.
    new_tags = tags.copy()
    new_tags[100:400] = 2
    new_tags[700:720] = 254
    prov.set_tags(100, new_tags[100:720])
    _check(prov, orc, 2, inmem_rows(typed, new_tags), ext, q, Knn(10, 50))
    prov.close()


def test_inmem_errors():
    typed, values, adj, deg, n, tags, ext = inmem_fixture("f32", 300, 16, seed=1)
    bad = tags.copy()
    bad[n] = 1  # a start point that is not readable
    with pytest.raises(ANNError) as e:
        InmemProvider(typed, adj, deg, n, bad, ext, Metric.L2)
    assert e.value.status == Status.INVALID_ARGUMENT
    prov = InmemProvider(typed, adj, deg, n, tags, ext, Metric.L2)
    with pytest.raises(ANNError) as e:
        prov.set_tags(n, [0])
    assert e.value.status == Status.INVALID_ARGUMENT
    with pytest.raises(ANNError) as e:
        prov.search(Knn(10, 40), typed[:2, :8])
    assert e.value.status == Status.DIMENSION_MISMATCH
    prov.close()
