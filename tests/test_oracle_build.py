"""CPU: graph construction — the oracle's restatement (oracle/build.cpp) against the
library's host builder (dk_build_vamana) and against the reference's construction baselines.

* The oracle restates the reference's insert rules (search record, occlude_list, back edges
  through add_edge_and_prune) independently of the library; with the same batch schedule both
  must produce the identical graph, for every metric and alpha schedule, and the oracle's graph
  must not depend on its thread count.
* The reference's one-by-one insert baselines (grid_insert.rs, `insert_*_single`) are replayed:
  the lattice is built with batches of one point (the reference's `insert`), then searched with
  k = L = 10.  Lattice distances are small integers, so many candidates tie.  The reference
  orders a prune pool with an unstable sort on distance alone (SortedNeighbors,
  diskann/src/graph/internal/sorted_neighbors.rs:26-40, Rust's `sort_unstable_by`), so the
  order of tied candidates, and with it which of several equally distant neighbours a list
  keeps, is an artefact of that sort; this build breaks ties by id.  The bar is therefore what
  does not depend on tie order: the exact list of result distances, the set of ids at every
  distance below the last one returned, and the hop count.
"""

import ctypes
import json
import os

import numpy as np
import pytest

from diskann_b200 import Metric, datasets, graph
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("metric,dim,alpha", [(Metric.L2, 64, 1.2), (Metric.INNER_PRODUCT, 96, 1.2),
                                              (Metric.COSINE, 48, 1.2),
                                              (Metric.COSINE_NORMALIZED, 100, 1.2),
                                              (Metric.L2, 32, 1.0), (Metric.L2, 45, 1.4)])
def test_oracle_build_equals_host_build(metric, dim, alpha):
    if metric == Metric.L2:
        base, _ = datasets.gaussian_mixture(5000, dim, 16, 8.0, seed=dim)
    else:
        base, _ = datasets.normalized_gaussian(5000, dim, seed=dim)
    kw = dict(pruned_degree=24, l_build=40, alpha=alpha, max_batch=512)
    v0, a0, d0, n0 = graph.build_vamana(base, metric=metric, **kw)
    v1, a1, d1, n1 = O.build_vamana(base, int(metric), **kw)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(d0, d1)
    np.testing.assert_array_equal(a0, a1)


def test_oracle_build_is_thread_count_invariant():
    base, _ = datasets.gaussian_mixture(4000, 32, 8, 6.0, seed=3)
    g1 = O.build_vamana(base, O.METRIC_L2, 20, 40, num_threads=1, max_batch=256)
    g4 = O.build_vamana(base, O.METRIC_L2, 20, 40, num_threads=4, max_batch=256)
    for x, y in zip(g1[:3], g4[:3]):
        np.testing.assert_array_equal(x, y)


def test_oracle_medoid_matches_library():
    base, _ = datasets.gaussian_mixture(3000, 24, 8, 5.0, seed=11)
    assert O.medoid(base) == graph.compute_medoid(base)


def _insert_cases():
    with open(os.path.join(GOLDEN, "grid_insert.json")) as f:
        return json.load(f)


def _lattice_one_by_one(dims, size, build):
    """The grid_insert.rs set-up: lattice rows, start point [size] * dim with no edges,
    max_degree 2 * dim, target degree max(2, 2 * dim - 2), L_build 100, alpha 1.2, one point per
    batch (the reference's `insert`)."""
    v, _, _, n = datasets.grid(dims, size)
    md = 2 * dims
    target = min(max(2, md - 2), md)
    adj = np.zeros((n + 1, md), np.uint32)
    deg = np.zeros(n + 1, np.uint32)
    if build == "oracle":
        p = O.BuildParams(target, md, 100, 1.2, target, 0, 1, 1)
        rc = O.lib().orc_build_vamana(O._ptr(v), dims, n, 1, dims, O.METRIC_L2, ctypes.byref(p),
                                      O._ptr(adj), md, O._ptr(deg))
        assert rc == 0
    else:
        from diskann_b200.index import _check

        p = graph.BuildParams(target, md, 100, 1.2, target, 0, 1, 1)
        _check(graph._lib().dk_build_vamana(v.ctypes.data, dims, n, 1, dims, int(Metric.L2),
                                            ctypes.byref(p), adj.ctypes.data, md, deg.ctypes.data))
    return v, adj, deg, n


@pytest.mark.parametrize("build", ["oracle", "library"])
@pytest.mark.parametrize("case", _insert_cases(), ids=lambda c: f"d{c['grid_dims']}s{c['grid_size']}")
def test_single_insert_baselines_up_to_tie_order(case, build):
    v, adj, deg, n = _lattice_one_by_one(case["grid_dims"], case["grid_size"], build)
    ix = O.OracleIndex(v, adj, deg, n, O.METRIC_L2)
    for s in case["searches"]:
        ids, dists, st = ix.search(np.array(s["query"], np.float32), 10, 10, 1)
        want_d = [r[1] for r in s["results"]]
        assert [float(x) for x in dists[0]] == want_d
        last = want_d[-1]
        got_inner = sorted(int(i) for i, d in zip(ids[0], dists[0]) if d < last)
        want_inner = sorted(r[0] for r in s["results"] if r[1] < last)
        assert got_inner == want_inner
        assert int(st[0]["hops"]) == s["hops"]
        assert int(st[0]["result_count"]) == s["num_results"]
