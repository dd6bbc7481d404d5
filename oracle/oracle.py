"""ctypes front-end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

The oracle (oracle.cpp) restates the reference's greedy beam search on the CPU.  Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, always as
the checker or the timed CPU baseline, never as the product path.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lock = threading.Lock()
_lib = None

METRIC_COSINE = 0
METRIC_INNER_PRODUCT = 1
METRIC_L2 = 2
METRIC_COSINE_NORMALIZED = 3

STRATEGY_FULL_PRECISION = 0
STRATEGY_HYBRID = 1
STRATEGY_QUANTIZED = 2

INVALID_ID = 0xFFFFFFFF


class _Index(ctypes.Structure):
    _fields_ = [
        ("num_points", ctypes.c_uint32),
        ("num_frozen", ctypes.c_uint32),
        ("dim", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("vectors", ctypes.c_void_p),
        ("vector_stride", ctypes.c_uint32),
        ("adjacency", ctypes.c_void_p),
        ("degrees", ctypes.c_void_p),
        ("adjacency_stride", ctypes.c_uint32),
        ("max_degree", ctypes.c_uint32),
        ("pq_chunks", ctypes.c_uint32),
        ("pq_offsets", ctypes.c_void_p),
        ("pq_pivots", ctypes.c_void_p),
        ("pq_codes", ctypes.c_void_p),
        ("pq_code_stride", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("cmps", ctypes.c_uint32),
        ("hops", ctypes.c_uint32),
        ("result_count", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
    ]


class BuildParams(ctypes.Structure):
    _fields_ = [
        ("pruned_degree", ctypes.c_uint32),
        ("max_degree", ctypes.c_uint32),
        ("l_build", ctypes.c_uint32),
        ("alpha", ctypes.c_float),
        ("max_backedges", ctypes.c_uint32),
        ("max_occlusion", ctypes.c_uint32),
        ("num_threads", ctypes.c_uint32),
        ("max_batch", ctypes.c_uint32),
    ]


STATS_DTYPE = np.dtype(
    [("cmps", np.uint32), ("hops", np.uint32), ("result_count", np.uint32), ("flags", np.uint32)]
)


def build() -> str:
    """Compile the oracle (g++) if it is missing or stale; return the library path."""
    src = [os.path.join(_HERE, f) for f in ("oracle.cpp", "build.cpp", "oracle.h", "Makefile")]
    if os.path.exists(_LIB_PATH) and all(
        os.path.getmtime(_LIB_PATH) >= os.path.getmtime(s) for s in src
    ):
        return _LIB_PATH
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_distance.restype = ctypes.c_float
            L.orc_distance.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]
            L.orc_validate_knn.restype = ctypes.c_int32
            L.orc_validate_knn.argtypes = [ctypes.c_uint32] * 3
            L.orc_search.restype = ctypes.c_int32
            L.orc_search_batch.restype = ctypes.c_int32
            L.orc_search_batch.argtypes = [
                ctypes.POINTER(_Index), ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint32,
                ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
            ]
            L.orc_bruteforce_f64.restype = None
            L.orc_bruteforce_f64.argtypes = [
                ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32,
                ctypes.c_void_p, ctypes.c_void_p,
            ]
            L.orc_build_vamana.restype = ctypes.c_int32
            L.orc_build_vamana.argtypes = [
                ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                ctypes.c_int32, ctypes.POINTER(BuildParams), ctypes.c_void_p, ctypes.c_uint32,
                ctypes.c_void_p]
            L.orc_medoid.restype = ctypes.c_uint32
            L.orc_medoid.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
            L.orc_pq_table.restype = None
            L.orc_pq_table.argtypes = [ctypes.POINTER(_Index), ctypes.c_void_p, ctypes.c_void_p]
            L.orc_range_search.restype = ctypes.c_int32
            L.orc_range_search.argtypes = [
                ctypes.POINTER(_Index), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_inmem_search.restype = ctypes.c_int32
            L.orc_inmem_search.argtypes = [
                ctypes.POINTER(_Index), ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_paged_create.restype = ctypes.c_int32
            L.orc_paged_create.argtypes = [ctypes.POINTER(_Index), ctypes.c_void_p, ctypes.c_uint32,
                                           ctypes.c_void_p, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_void_p)]
            L.orc_paged_next.restype = ctypes.c_int32
            L.orc_paged_next.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_paged_destroy.restype = None
            L.orc_paged_destroy.argtypes = [ctypes.c_void_p]
            _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def distance(metric: int, x: np.ndarray, y: np.ndarray) -> float:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    assert x.shape == y.shape
    return float(lib().orc_distance(metric, _ptr(x), _ptr(y), x.size))


class OracleIndex:
    """CPU oracle over host arrays laid out as the GPU index's inputs.

    ``vectors``: (N + F, D) float32; ``adjacency``: (N + F, S) uint32 with ``degrees`` (N + F,)
    giving each list's length; ids N..N+F-1 are the frozen start points.
    """

    def __init__(self, vectors, adjacency, degrees, num_points, metric,
                 pq_offsets=None, pq_pivots=None, pq_codes=None):
        self.vectors = np.ascontiguousarray(vectors, dtype=np.float32)
        self.adjacency = np.ascontiguousarray(adjacency, dtype=np.uint32)
        self.degrees = np.ascontiguousarray(degrees, dtype=np.uint32)
        total = self.vectors.shape[0]
        assert self.adjacency.shape[0] == total and self.degrees.shape[0] == total
        self.num_points = int(num_points)
        self.num_frozen = total - self.num_points
        self.dim = self.vectors.shape[1]
        self.metric = int(metric)
        self.pq_offsets = None if pq_offsets is None else np.ascontiguousarray(pq_offsets, dtype=np.uint32)
        self.pq_pivots = None if pq_pivots is None else np.ascontiguousarray(pq_pivots, dtype=np.float32)
        self.pq_codes = None if pq_codes is None else np.ascontiguousarray(pq_codes, dtype=np.uint8)
        s = _Index()
        s.num_points = self.num_points
        s.num_frozen = self.num_frozen
        s.dim = self.dim
        s.metric = self.metric
        s.vectors = _ptr(self.vectors)
        s.vector_stride = self.dim
        s.adjacency = _ptr(self.adjacency)
        s.degrees = _ptr(self.degrees)
        s.adjacency_stride = self.adjacency.shape[1]
        s.max_degree = self.adjacency.shape[1]
        if self.pq_codes is not None:
            s.pq_chunks = len(self.pq_offsets) - 1
            s.pq_offsets = _ptr(self.pq_offsets)
            s.pq_pivots = _ptr(self.pq_pivots)
            s.pq_codes = _ptr(self.pq_codes)
            s.pq_code_stride = self.pq_codes.shape[1]
        self._s = s

    def search(self, queries, k, l, beam_width=1, strategy=STRATEGY_FULL_PRECISION, threads=1):
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), dtype=np.uint32)
        dists = np.empty((nq, k), dtype=np.float32)
        stats = np.zeros(nq, dtype=STATS_DTYPE)
        rc = lib().orc_search_batch(
            ctypes.byref(self._s), strategy, _ptr(q), q.shape[1], nq, k, l, beam_width,
            _ptr(ids), _ptr(dists), _ptr(stats), threads,
        )
        if rc != 0:
            raise ValueError(f"oracle search failed with status {rc}")
        return ids, dists, stats

    def range_search(self, query, starting_l, radius, beam_width=1, inner_radius=None,
                     initial_slack=1.0, range_slack=1.0, max_returned=0, capacity=None):
        """Range search of one query (range_search.rs restated); returns ``(ids, dists, stats)``
        with the results that passed the filter (stats["flags"] bit 1: second round ran)."""
        q = np.ascontiguousarray(np.ravel(query), dtype=np.float32)
        cap = capacity if capacity is not None else (max_returned or self.num_points)
        ids = np.empty(max(cap, 1), dtype=np.uint32)
        dists = np.empty(max(cap, 1), dtype=np.float32)
        st = np.zeros(1, dtype=STATS_DTYPE)
        rc = lib().orc_range_search(
            ctypes.byref(self._s), _ptr(q), starting_l, beam_width, radius,
            float("nan") if inner_radius is None else inner_radius, initial_slack, range_slack,
            max_returned, cap, _ptr(ids), _ptr(dists), _ptr(st))
        if rc != 0:
            raise ValueError(f"oracle range search failed with status {rc}")
        n = int(st[0]["result_count"])
        return ids[:n], dists[:n], st[0]

    def inmem_search(self, elem, rows, external_ids, query, k, l, beam_width=1):
        """diskann-inmem search of one query (provider.rs restated).  ``rows``: the store's
        slots (uint8, element bytes then the tag); ``elem``: 0 f32, 1 f16, 2 u8, 3 i8; the
        index's own vectors must hold the rows' f32 values.  ``query``: f32 values for f32 /
        f16 data, the element bytes for u8 / i8.  Returns ``(external ids, dists, stats)``."""
        rows = np.ascontiguousarray(rows, dtype=np.uint8)
        ext = np.ascontiguousarray(external_ids, dtype=np.uint64)
        if elem in (2, 3):
            q = np.ascontiguousarray(np.ravel(query)).view(np.uint8).copy()
        else:
            q = np.ascontiguousarray(np.ravel(query), dtype=np.float32)
        ids = np.empty(k, dtype=np.uint64)
        dists = np.empty(k, dtype=np.float32)
        st = np.zeros(1, dtype=STATS_DTYPE)
        rc = lib().orc_inmem_search(ctypes.byref(self._s), elem, _ptr(rows), rows.shape[1],
                                    _ptr(ext), _ptr(q), k, l, beam_width, _ptr(ids), _ptr(dists),
                                    _ptr(st))
        if rc != 0:
            raise ValueError(f"oracle inmem search failed with status {rc}")
        return ids, dists, st[0]

    def paged_search(self, query, l_value, init_ids=None):
        """Start a paged search of one query (paged.rs restated); returns an
        :class:`OraclePagedSearch` whose ``next_page(k)`` yields ``(ids, dists, stats)``."""
        return OraclePagedSearch(self, query, l_value, init_ids)

    def pq_table(self, query):
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty((len(self.pq_offsets) - 1, 256), dtype=np.float32)
        lib().orc_pq_table(ctypes.byref(self._s), _ptr(q), _ptr(out))
        return out


class OraclePagedSearch:
    """One paged-search session (index.rs:2101-2160, paged.rs:52-151); stats are the
    session's running comparison and hop counters."""

    def __init__(self, index: "OracleIndex", query, l_value: int, init_ids=None):
        self._index = index  # keeps the index arrays alive
        q = np.ascontiguousarray(np.ravel(query), dtype=np.float32)
        init = None if init_ids is None else np.ascontiguousarray(init_ids, dtype=np.uint32)
        h = ctypes.c_void_p()
        rc = lib().orc_paged_create(ctypes.byref(index._s), _ptr(q), l_value, _ptr(init),
                                    0 if init is None else init.size, ctypes.byref(h))
        if rc != 0:
            raise ValueError(f"oracle paged search failed with status {rc}")
        self._h = h

    def next_page(self, k: int):
        ids = np.empty(max(k, 1), dtype=np.uint32)
        dists = np.empty(max(k, 1), dtype=np.float32)
        n = np.zeros(1, dtype=np.uint32)
        st = np.zeros(1, dtype=STATS_DTYPE)
        rc = lib().orc_paged_next(self._h, k, _ptr(ids), _ptr(dists), _ptr(n), _ptr(st))
        if rc != 0:
            raise ValueError(f"oracle paged search failed with status {rc}")
        return ids[: n[0]], dists[: n[0]], st[0]

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_paged_destroy(self._h)
            self._h = None


def validate_knn(k: int, l: int, beam_width: int) -> int:
    return int(lib().orc_validate_knn(k, l, beam_width))


def bruteforce_f64(base, queries, k, metric):
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
    ids = np.empty((q.shape[0], k), dtype=np.uint32)
    d = np.empty((q.shape[0], k), dtype=np.float64)
    lib().orc_bruteforce_f64(_ptr(base), base.shape[0], base.shape[1], base.shape[1], _ptr(q),
                             q.shape[0], k, metric, _ptr(ids), _ptr(d))
    return ids, d


def medoid(base) -> int:
    """The reference's medoid rule (medoid.rs:15-45) restated (build.cpp)."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    return int(lib().orc_medoid(_ptr(base), base.shape[1], base.shape[0], base.shape[1]))


def build_vamana(base, metric, pruned_degree, l_build, alpha=1.2, max_degree=None,
                 backedge_ratio=1.0, num_threads=0, max_batch=0):
    """Graph construction restated on the CPU (build.cpp), with the medoid row copied to the
    frozen start point (id N).  Returns ``(vectors, adjacency, degrees, n)`` in the layout of
    ``diskann_b200.graph.build_vamana``, whose result it must equal."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    n, dim = base.shape
    med = medoid(base)
    vectors = np.vstack([base, base[med:med + 1]])
    md = max_degree or int(np.float32(pruned_degree) * np.float32(1.3))
    adjacency = np.zeros((n + 1, md), np.uint32)
    degrees = np.zeros(n + 1, np.uint32)
    p = BuildParams(pruned_degree, md, l_build, alpha, int(np.ceil(backedge_ratio * pruned_degree)),
                    0, num_threads, max_batch)
    rc = lib().orc_build_vamana(_ptr(vectors), dim, n, 1, dim, int(metric), ctypes.byref(p),
                                _ptr(adjacency), md, _ptr(degrees))
    if rc != 0:
        raise ValueError(f"oracle build failed with status {rc}")
    return vectors, adjacency, degrees, n
