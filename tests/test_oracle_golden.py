"""CPU: pin the oracle against the reference's golden vectors and basic invariants."""

import json
import os

import numpy as np
import pytest

from diskann_b200 import datasets
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _grid_cases():
    with open(os.path.join(GOLDEN, "grid_search.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _grid_cases(),
                         ids=lambda c: f"d{c['grid_dims']}s{c['grid_size']}b{c['beam_width']}q{c['query'][0]:g}")
def test_oracle_matches_grid_golden(case):
    """Exact ids, distances, comparisons and hops of grid_search.rs's baselines."""
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    ix = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    ids, dists, st = ix.search(np.array(case["query"], np.float32), case["k"], case["l"],
                               case["beam_width"])
    assert [int(i) for i in ids[0]] == [r[0] for r in case["results"]]
    assert [float(x) for x in dists[0]] == [r[1] for r in case["results"]]
    assert int(st[0]["cmps"]) == case["comparisons"]
    assert int(st[0]["hops"]) == case["hops"]
    assert int(st[0]["result_count"]) == case["num_results"]


def test_flat_golden_bruteforce():
    """The f64 brute force reproduces flat_knn_search's ground truth (as distance lists;
    ties may be listed in another order)."""
    with open(os.path.join(GOLDEN, "flat_knn_search.json")) as f:
        cases = json.load(f)
    for c in cases:
        v, _, _, n = datasets.grid(c["grid_dims"], c["grid_size"])
        ids, d = O.bruteforce_f64(v[:n], np.array(c["query"], np.float32), c["k"], O.METRIC_L2)
        cnt = c["result_count"]
        gt = c["ground_truth"]
        assert [float(x) for x in d[0][:cnt]] == [g[1] for g in gt]
        # Same id sets within each distance value.
        for dist in set(g[1] for g in gt):
            exp = {g[0] for g in gt if g[1] == dist}
            got = {int(i) for i, x in zip(ids[0][:cnt], d[0][:cnt]) if x == dist}
            if dist != max(g[1] for g in gt):
                assert exp == got


@pytest.mark.parametrize("k,l,bw,status", [(0, 10, 1, 1), (1, 0, 1, 2), (11, 10, 1, 3),
                                           (10, 10, 0, 4), (10, 10, 1, 0)])
def test_oracle_knn_validation(k, l, bw, status):
    assert O.validate_knn(k, l, bw) == status


@pytest.mark.parametrize("dim", [1, 3, 7, 8, 13, 32, 40, 96, 100, 128, 384, 768])
def test_oracle_distances_close_to_f64(dim):
    rng = np.random.default_rng(dim)
    x = rng.standard_normal(dim).astype(np.float32)
    y = rng.standard_normal(dim).astype(np.float32)
    x64, y64 = x.astype(np.float64), y.astype(np.float64)
    l2 = ((x64 - y64) ** 2).sum()
    ip = (x64 * y64).sum()
    cos = ip / np.sqrt((x64 * x64).sum() * (y64 * y64).sum())
    assert O.distance(O.METRIC_L2, x, y) == pytest.approx(l2, rel=1e-5)
    assert O.distance(O.METRIC_INNER_PRODUCT, x, y) == pytest.approx(-ip, rel=1e-4, abs=1e-4)
    assert O.distance(O.METRIC_COSINE, x, y) == pytest.approx(1 - cos, rel=1e-4, abs=1e-5)
    assert O.distance(O.METRIC_COSINE_NORMALIZED, x, y) == pytest.approx(1 - ip, rel=1e-4, abs=1e-4)


def test_oracle_cosine_zero_norm():
    """A norm below f32::MIN_POSITIVE gives similarity 0 (simd.rs:2355-2357)."""
    x = np.zeros(16, np.float32)
    y = np.ones(16, np.float32)
    assert O.distance(O.METRIC_COSINE, x, y) == 1.0


def test_oracle_pq_table_matches_direct():
    """ADC lookup equals the sum of per-chunk direct distances (pq/distance/dynamic.rs tests)."""
    from tests.helpers import random_index, simple_pq

    v, a, d, n = random_index(300, 32, 8, seed=3)
    off, piv, codes = simple_pq(v, 8, seed=4)
    ix = O.OracleIndex(v, a, d, n, O.METRIC_L2, off, piv, codes)
    q = v[5] + 0.5
    table = ix.pq_table(q)
    for m in range(8):
        s, e = off[m], off[m + 1]
        for c in (0, 17, 255):
            ref = float(((q[s:e].astype(np.float64) - piv[c, s:e]) ** 2).sum())
            assert table[m, c] == pytest.approx(ref, rel=1e-5, abs=1e-6)


def test_oracle_search_finds_exact_on_complete_graph():
    """With a complete graph and L >= N every point is scored, so results are exact."""
    rng = np.random.default_rng(0)
    n, dim = 40, 8
    base = rng.standard_normal((n, dim)).astype(np.float32)
    vectors = np.vstack([base, base[:1]])
    adj = np.array([[j for j in range(n + 1) if j != i][: n] for i in range(n + 1)], np.uint32)
    deg = np.full(n + 1, n, np.uint32)
    ix = O.OracleIndex(vectors, adj, deg, n, O.METRIC_L2)
    q = rng.standard_normal(dim).astype(np.float32)
    ids, dists, st = ix.search(q, 5, 50)
    gt, _ = O.bruteforce_f64(base, q, 5, O.METRIC_L2)
    assert list(ids[0]) == list(gt[0])
    assert st[0]["cmps"] == n + 1


# ---------------------------------------------------------------------------------------
# The x86-64-v3 accumulation orders, restated independently in numpy (float32 rounding after
# every operation; fma emulated in float64, exact for these inputs up to a double rounding
# that is vanishingly rare), against the oracle's distance function bit for bit.
# ---------------------------------------------------------------------------------------

def _f32(x):
    return np.float32(x)


def _fma(a, b, c):
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def _sum_tree(t):
    q = [_f32(t[i] + t[i + 4]) for i in range(4)]
    return _f32(_f32(q[0] + q[2]) + _f32(q[1] + q[3]))


def _strategy_4x1(x, y, l2):
    """L2 / IP on V3: Strategy4x1 (simd.rs:321-363), then the masked remainder."""
    n = len(x)
    s = np.zeros((4, 8), np.float32)
    trip, k = n // 32, 0
    for k in range(trip * 4 + (n - 32 * trip) // 8):
        j = k % 4 if k < 4 * trip else (k - 4 * trip)
        for lane in range(8):
            e = 8 * k + lane
            c = _f32(x[e] - y[e]) if l2 else None
            s[j][lane] = _fma(c, c, s[j][lane]) if l2 else _fma(x[e], y[e], s[j][lane])
    t = [_f32(_f32(s[0][i] + s[1][i]) + _f32(s[2][i] + s[3][i])) for i in range(8)]
    base = n - n % 8
    for lane in range(n % 8):
        e = base + lane
        if l2:
            c = _f32(x[e] - y[e])
            t[lane] = _fma(c, c, t[lane])
        else:
            t[lane] = _fma(x[e], y[e], t[lane])
    return _sum_tree(t)


def _cosine_2x4(x, y):
    """CosineStateless on V3: Strategy2x4 (simd.rs:422-482), masked remainder, then `sum`."""
    n = len(x)
    acc = np.zeros((3, 2, 8), np.float32)
    for k in range(n // 8):
        for lane in range(8):
            a, b = x[8 * k + lane], y[8 * k + lane]
            acc[0][k % 2][lane] = _fma(a, a, acc[0][k % 2][lane])
            acc[1][k % 2][lane] = _fma(b, b, acc[1][k % 2][lane])
            acc[2][k % 2][lane] = _fma(a, b, acc[2][k % 2][lane])
    t = [[_f32(acc[q][0][i] + acc[q][1][i]) for i in range(8)] for q in range(3)]
    base = n - n % 8
    for lane in range(n % 8):
        a, b = x[base + lane], y[base + lane]
        t[0][lane] = _fma(a, a, t[0][lane])
        t[1][lane] = _fma(b, b, t[1][lane])
        t[2][lane] = _fma(a, b, t[2][lane])
    nx, ny, xy = _sum_tree(t[0]), _sum_tree(t[1]), _sum_tree(t[2])
    if nx < 1.17549435e-38 or ny < 1.17549435e-38:
        sim = np.float32(0.0)
    else:
        den = _f32(_f32(np.sqrt(nx)) * _f32(np.sqrt(ny)))
        sim = np.float32(max(-1.0, min(1.0, float(_f32(xy / den)))))
    return _f32(np.float32(1.0) - sim)


@pytest.mark.parametrize("n", [1, 5, 8, 13, 16, 24, 31, 32, 33, 40, 56, 96, 100, 128, 200, 384])
def test_oracle_accumulation_orders(n):
    rng = np.random.default_rng(n)
    for trial in range(3):
        scale = np.float32(10.0 ** rng.uniform(-2, 2))
        x = (rng.standard_normal(n) * scale).astype(np.float32)
        y = (rng.standard_normal(n) * scale).astype(np.float32)
        got_l2 = np.float32(O.distance(O.METRIC_L2, x, y))
        got_ip = np.float32(O.distance(O.METRIC_INNER_PRODUCT, x, y))
        got_cos = np.float32(O.distance(O.METRIC_COSINE, x, y))
        assert got_l2.view(np.uint32) == _strategy_4x1(x, y, True).view(np.uint32)
        assert got_ip.view(np.uint32) == np.float32(-_strategy_4x1(x, y, False)).view(np.uint32)
        assert got_cos.view(np.uint32) == _cosine_2x4(x, y).view(np.uint32)


def _direct_cosine(q, pivots, offsets, code):
    """DirectCosine (fixed_chunk_pq_table.rs:32-56, 233-243): per chunk one CosineStateless
    pass from zero, folded lane by lane into the running accumulator, then `sum`."""
    total = np.zeros((3, 8), np.float32)
    for m in range(len(offsets) - 1):
        a0, a1 = int(offsets[m]), int(offsets[m + 1])
        x, y = q[a0:a1], pivots[int(code[m])][a0:a1]
        n = len(x)
        acc = np.zeros((3, 2, 8), np.float32)
        for k in range(n // 8):
            for lane in range(8):
                a, b = x[8 * k + lane], y[8 * k + lane]
                acc[0][k % 2][lane] = _fma(a, a, acc[0][k % 2][lane])
                acc[1][k % 2][lane] = _fma(b, b, acc[1][k % 2][lane])
                acc[2][k % 2][lane] = _fma(a, b, acc[2][k % 2][lane])
        t = [[_f32(acc[i][0][j] + acc[i][1][j]) for j in range(8)] for i in range(3)]
        base = n - n % 8
        for lane in range(n % 8):
            a, b = x[base + lane], y[base + lane]
            t[0][lane] = _fma(a, a, t[0][lane])
            t[1][lane] = _fma(b, b, t[1][lane])
            t[2][lane] = _fma(a, b, t[2][lane])
        for i in range(3):
            for j in range(8):
                total[i][j] = _f32(total[i][j] + t[i][j])
    nx, ny, xy = _sum_tree(total[0]), _sum_tree(total[1]), _sum_tree(total[2])
    if nx < 1.17549435e-38 or ny < 1.17549435e-38:
        sim = np.float32(0.0)
    else:
        den = _f32(_f32(np.sqrt(nx)) * _f32(np.sqrt(ny)))
        sim = np.float32(max(-1.0, min(1.0, float(_f32(xy / den)))))
    return _f32(np.float32(1.0) - sim)


@pytest.mark.parametrize("dim,chunks", [(64, 16), (100, 7), (128, 8)])
def test_oracle_pq_direct_cosine(dim, chunks):
    """The oracle's Quantized search with the Cosine metric returns DirectCosine distances."""
    rng = np.random.default_rng(dim)
    n = 40
    base = rng.standard_normal((n, dim)).astype(np.float32)
    vectors = np.vstack([base, base[:1]])
    adj = np.array([[j for j in range(n + 1) if j != i][:n] for i in range(n + 1)], np.uint32)
    deg = np.full(n + 1, n, np.uint32)
    offsets = np.linspace(0, dim, chunks + 1).round().astype(np.uint32)
    pivots = rng.standard_normal((256, dim)).astype(np.float32)
    codes = rng.integers(0, 256, size=(n + 1, chunks)).astype(np.uint8)
    orc = O.OracleIndex(vectors, adj, deg, n, O.METRIC_COSINE, offsets, pivots, codes)
    q = rng.standard_normal((3, dim)).astype(np.float32)
    ids, dists, _ = orc.search(q, 10, 20, 1, O.STRATEGY_QUANTIZED)
    for i in range(q.shape[0]):
        for j in range(10):
            want = _direct_cosine(q[i], pivots, offsets, codes[ids[i, j]])
            assert dists[i, j].view(np.uint32) == want.view(np.uint32)


def _range_cases():
    with open(os.path.join(GOLDEN, "range_search.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _range_cases(), ids=lambda c: c["source"].split("/")[-1][:-5])
def test_oracle_matches_range_golden(case):
    """Exact results, comparisons, hops and second-round flag of range_search.rs's baselines."""
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    ix = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    ids, dists, st = ix.range_search(
        np.array(case["query"], np.float32), case["starting_l"], case["radius"],
        inner_radius=case["inner_radius"], initial_slack=case["initial_slack"],
        range_slack=case["range_slack"], max_returned=case["max_returned"] or 0)
    assert [[int(i), float(x)] for i, x in zip(ids, dists)] == case["results"]
    assert int(st["cmps"]) == case["comparisons"]
    assert int(st["hops"]) == case["hops"]
    assert int(st["result_count"]) == case["result_count"]
    assert bool(int(st["flags"]) & 2) == case["second_round"]


def _paged_cases():
    with open(os.path.join(GOLDEN, "paged_search.json")) as f:
        return json.load(f)


def _oracle_pages(ix, case):
    ps = ix.paged_search(np.array(case["query"], np.float32), case["search_l"])
    pages = []
    while True:
        ids, dists, _ = ps.next_page(case["page_size"])
        if len(ids) == 0:
            break
        pages.append([[int(i), float(x)] for i, x in zip(ids, dists)])
    return pages, ps


@pytest.mark.parametrize("case", _paged_cases(), ids=lambda c: c["source"].split("/")[-1][:-5])
def test_oracle_matches_paged_golden(case):
    """Every page of paged_search.rs's baselines (ids and distances, in order), until the
    search is exhausted; then further calls stay empty."""
    v, a, d, n = datasets.grid(case["grid_dims"], case["grid_size"])
    ix = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    pages, ps = _oracle_pages(ix, case)
    assert pages == case["pages"]
    assert sum(len(p) for p in pages) == case["total_results"]
    assert len(ps.next_page(case["page_size"])[0]) == 0


def test_oracle_paged_errors():
    v, a, d, n = datasets.grid(3, 5)
    ps = O.OracleIndex(v, a, d, n, O.METRIC_L2).paged_search(np.full(3, 5.0, np.float32), 8)
    for k in (0, 9):
        with pytest.raises(ValueError):
            ps.next_page(k)


def test_oracle_rerank_sorts_nan_last():
    """Hybrid rerank order in the oracle: ascending exact distance, NaN distances (rows with a
    NaN coordinate, reachable through their finite PQ codes) after every number."""
    from tests.helpers import random_index, simple_pq

    v, a, d, n = random_index(600, 16, 12, seed=81, max_degree=12)
    off, piv, codes = simple_pq(v, 4, seed=82)
    v[:n][np.arange(n) % 3 != 0, 5] = np.nan
    ix = O.OracleIndex(v, a, d, n, O.METRIC_L2, off, piv, codes)
    q = np.nan_to_num(v[:8]) + 0.25
    ids, dists, stats = ix.search(q, 40, 100, 1, O.STRATEGY_HYBRID)
    saw_nan = False
    for row, cnt in zip(dists, stats["result_count"]):
        row = row[:cnt]
        nan = np.isnan(row)
        first = int(np.argmax(nan)) if nan.any() else len(row)
        assert not nan[:first].any() and nan[first:].all()
        assert (np.diff(row[:first]) >= 0).all()
        saw_nan |= bool(nan.any())
    assert saw_nan
