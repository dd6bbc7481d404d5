"""Host-side mirror of the reference's search surface over the C ABI.

Reference shapes mirrored here (paths relative to the reference repository):

* ``Knn`` — diskann/src/graph/search/knn_search.rs:76-119 (k, L, beam width; validation and
  the ``KnnSearchError`` kinds).
* ``Metric`` — diskann-vector/src/distance/metric.rs:11-52 (same integer codes).
* ``FullPrecision`` / ``Hybrid`` / ``Quantized`` — the in-memory strategies
  (diskann-providers/.../inmem/full_precision.rs:476-506, inmem/product.rs:363-394, 537-566).
* ``GpuProvider`` — the device-resident counterpart of ``DefaultProvider``
  (inmem/provider.rs:227-352): vectors, optional PQ codes, fixed-slot adjacency and frozen
  start points with ids ``num_points..num_points+F-1``.
* ``DiskANNIndex.search`` — ``DiskANNIndex::search`` (diskann/src/graph/index.rs:2034-2070),
  batched: it returns ids, distances and per-query ``SearchStats`` (index.rs:90-102).
"""

from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass

import numpy as np

from . import _native

STATS_DTYPE = np.dtype(
    [("cmps", np.uint32), ("hops", np.uint32), ("result_count", np.uint32), ("flags", np.uint32)]
)
INVALID_ID = 0xFFFFFFFF


class Metric(enum.IntEnum):
    COSINE = 0
    INNER_PRODUCT = 1
    L2 = 2
    COSINE_NORMALIZED = 3


class Status(enum.IntEnum):
    OK = 0
    K_ZERO = 1
    L_ZERO = 2
    L_LESS_THAN_K = 3
    BEAM_WIDTH_ZERO = 4
    NO_PQ = 5
    INVALID_ARGUMENT = 6
    INVALID_GRAPH = 7
    DIMENSION_MISMATCH = 8
    OUT_OF_MEMORY = 9
    CUDA = 10
    DEVICE_TIMEOUT = 11
    UNSUPPORTED = 12
    ADMISSION = 13
    CANCELLED = 14
    NOT_FOUND = 15
    NO_LOW_PRECISION = 16
    NOT_READY = 17


class ANNError(RuntimeError):
    """An error returned by the C ABI (the reference's ``ANNError``)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{Status(status).name}: {message}")
        self.status = Status(status)
        self.message = message


class KnnSearchError(ANNError, ValueError):
    """Invalid ``Knn`` parameters (knn_search.rs:39-44)."""


def _check(status: int) -> None:
    if status != 0:
        st, msg = _native.last_error()
        cls = KnnSearchError if status in (1, 2, 3, 4) else ANNError
        raise cls(status, msg if st == status else "")


class Knn:
    """k-NN search parameters: ``Knn(k_value, l_value, beam_width=None)``."""

    def __init__(self, k_value: int, l_value: int, beam_width: int | None = None):
        bw = 1 if beam_width is None else int(beam_width)
        if k_value == 0:
            raise KnnSearchError(Status.K_ZERO, "k_value must be nonzero")
        if l_value == 0:
            raise KnnSearchError(Status.L_ZERO, "l_value must be nonzero")
        if k_value > l_value:
            raise KnnSearchError(
                Status.L_LESS_THAN_K, f"l_value ({l_value}) cannot be less than k_value ({k_value})"
            )
        if bw == 0:
            raise KnnSearchError(Status.BEAM_WIDTH_ZERO, "beam width must be nonzero")
        self.k_value = int(k_value)
        self.l_value = int(l_value)
        self.beam_width = bw

    def __repr__(self) -> str:
        return f"Knn(k={self.k_value}, l={self.l_value}, beam_width={self.beam_width})"


class Range:
    """Range search parameters (range_search.rs:63-110): ``Range(starting_l, radius,
    beam_width=None, inner_radius=None, initial_slack=1.0, range_slack=1.0,
    max_returned=None)``."""

    def __init__(self, starting_l: int, radius: float, beam_width: int | None = None,
                 inner_radius: float | None = None, initial_slack: float = 1.0,
                 range_slack: float = 1.0, max_returned: int | None = None):
        bw = 1 if beam_width is None else int(beam_width)
        if bw == 0:
            raise KnnSearchError(Status.BEAM_WIDTH_ZERO, "beam width cannot be zero")
        if starting_l == 0:
            raise KnnSearchError(Status.L_ZERO, "l_value cannot be zero")
        if max_returned is not None and max_returned < starting_l:
            raise ANNError(Status.INVALID_ARGUMENT,
                           "max_returned must be greater than or equal to starting_l")
        if not 0.0 <= initial_slack <= 1.0:
            raise ANNError(Status.INVALID_ARGUMENT, "initial_search_slack must be between 0 and 1.0")
        if range_slack < 1.0:
            raise ANNError(Status.INVALID_ARGUMENT,
                           "range_search_slack must be greater than or equal to 1.0")
        if inner_radius is not None and inner_radius > radius:
            raise ANNError(Status.INVALID_ARGUMENT, "inner_radius must be less than or equal to radius")
        self.starting_l = int(starting_l)
        self.radius = float(radius)
        self.beam_width = bw
        self.inner_radius = inner_radius
        self.initial_slack = float(initial_slack)
        self.range_slack = float(range_slack)
        self.max_returned = max_returned


class _Strategy:
    code = -1

    def __repr__(self) -> str:
        return type(self).__name__ + "()"


class FullPrecision(_Strategy):
    """FP32 traversal; FilterStartPoints + copy."""

    code = 0


class Hybrid(_Strategy):
    """PQ (ADC) traversal; FilterStartPoints + exact full-precision Rerank."""

    code = 1


class Quantized(_Strategy):
    """PQ (ADC) traversal; FilterStartPoints + copy."""

    code = 2


class BF16(_Strategy):
    """Traversal scored from BF16 rows (FP32 accumulation); FilterStartPoints + exact FP32
    Rerank.  Needs a provider created with ``low_precision=("bf16",)``."""

    code = 3


class FP8(_Strategy):
    """Traversal scored from FP8-E4M3 rows with a per-vector FP32 scale (FP32 accumulation);
    FilterStartPoints + exact FP32 Rerank.  Needs ``low_precision=("fp8",)``."""

    code = 4


@dataclass
class PQData:
    """Product quantisation schema and codes (FixedChunkPQTable layout)."""

    offsets: np.ndarray  # (M+1,) uint32
    pivots: np.ndarray  # (256, D) float32
    codes: np.ndarray  # (N+F, M) uint8


class GpuProvider:
    """Device-resident in-memory provider built from host arrays.

    ``vectors`` (N+F, D) float32, ``adjacency`` (N+F, S) uint32 with ``degrees`` (N+F,);
    rows ``num_points..`` are frozen start points.
    """

    def __init__(self, vectors, adjacency, degrees, num_points: int, metric=Metric.L2,
                 pq: PQData | None = None, device: int = 0, low_precision=()):
        L = _native.load()
        vectors = np.ascontiguousarray(vectors, dtype=np.float32)
        adjacency = np.ascontiguousarray(adjacency, dtype=np.uint32)
        degrees = np.ascontiguousarray(degrees, dtype=np.uint32)
        d = _native.IndexDesc()
        d.num_points = int(num_points)
        d.num_frozen = vectors.shape[0] - int(num_points)
        d.dim = vectors.shape[1]
        d.metric = int(metric)
        d.vectors = vectors.ctypes.data
        d.vector_stride = vectors.shape[1]
        d.adjacency = adjacency.ctypes.data
        d.adjacency_stride = adjacency.shape[1]
        d.degrees = degrees.ctypes.data
        d.max_degree = adjacency.shape[1]
        flags = 0
        for lp in low_precision:
            flags |= {"bf16": _native.INDEX_BF16, "fp8": _native.INDEX_FP8}[lp]
        d.flags = flags
        keep = [vectors, adjacency, degrees]
        if pq is not None:
            off = np.ascontiguousarray(pq.offsets, dtype=np.uint32)
            piv = np.ascontiguousarray(pq.pivots, dtype=np.float32)
            codes = np.ascontiguousarray(pq.codes, dtype=np.uint8)
            d.pq_chunks = len(off) - 1
            d.pq_offsets = off.ctypes.data
            d.pq_pivots = piv.ctypes.data
            d.pq_codes = codes.ctypes.data
            d.pq_code_stride = codes.shape[1]
            keep += [off, piv, codes]
        handle = ctypes.c_void_p()
        _check(L.dk_index_create(ctypes.byref(d), int(device), ctypes.byref(handle)))
        del keep
        self._handle = handle
        self.num_points = int(num_points)
        self.num_frozen = int(d.num_frozen)
        self.dim = int(d.dim)
        self.metric = Metric(int(metric))
        self.device = int(device)
        self.has_pq = pq is not None

    @property
    def handle(self):
        if self._handle is None:
            raise ANNError(Status.INVALID_ARGUMENT, "provider is closed")
        return self._handle

    def info(self) -> dict:
        inf = _native.IndexInfo()
        _check(_native.load().dk_index_get_info(self.handle, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in inf._fields_}

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None:
            _native.load().dk_index_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# diskann-inmem store (diskann-inmem/src/store.rs, tag.rs): element types and tags.
ELEM_TYPES = {"f32": (0, np.float32), "f16": (1, np.float16), "u8": (2, np.uint8),
              "i8": (3, np.int8)}
TAG_AVAILABLE, TAG_OWNED, TAG_RETIRING, TAG_PUBLISHED, TAG_FROZEN = 0, 1, 2, 254, 255
NO_EXTERNAL_ID = 0xFFFFFFFFFFFFFFFF


def inmem_rows(vectors, tags) -> np.ndarray:
    """Store slots as the diskann-inmem store lays them out (store.rs:150-260): each row's
    element bytes, then its one-byte tag, padded to a multiple of 32 bytes."""
    v = np.ascontiguousarray(vectors)
    raw = v.view(np.uint8).reshape(v.shape[0], -1)
    stride = -(-(raw.shape[1] + 1) // 32) * 32
    rows = np.zeros((v.shape[0], stride), dtype=np.uint8)
    rows[:, : raw.shape[1]] = raw
    rows[:, raw.shape[1]] = np.asarray(tags, dtype=np.uint8)
    return rows


class InmemProvider:
    """The diskann-inmem provider's store on the GPU (``dk_inmem_index_create``).

    ``vectors``: (capacity + F, D) of the element type (float32 / float16 / uint8 / int8),
    the last F rows the frozen start points; ``tags``: per slot (``TAG_PUBLISHED`` /
    ``TAG_FROZEN`` readable, anything else not); ``external_ids``: per slot (uint64,
    ``NO_EXTERNAL_ID`` = none).  ``search`` runs the provider's search with its Translate
    post-processor and returns external ids.
    """

    def __init__(self, vectors, adjacency, degrees, capacity: int, tags, external_ids,
                 metric=Metric.L2, device: int = 0):
        v = np.ascontiguousarray(vectors)
        elem = next((code for code, dt in ELEM_TYPES.values() if v.dtype == dt), None)
        if elem is None:
            raise ANNError(Status.INVALID_ARGUMENT, f"unsupported element type {v.dtype}")
        rows = inmem_rows(v, tags)
        adjacency = np.ascontiguousarray(adjacency, dtype=np.uint32)
        degrees = np.ascontiguousarray(degrees, dtype=np.uint32)
        ext = np.ascontiguousarray(external_ids, dtype=np.uint64)
        d = _native.InmemDesc()
        d.capacity = int(capacity)
        d.num_frozen = v.shape[0] - int(capacity)
        d.dim = v.shape[1]
        d.metric = int(metric)
        d.elem = elem
        d.rows = rows.ctypes.data
        d.row_stride = rows.shape[1]
        d.adjacency = adjacency.ctypes.data
        d.adjacency_stride = adjacency.shape[1]
        d.degrees = degrees.ctypes.data
        d.max_degree = adjacency.shape[1]
        d.external_ids = ext.ctypes.data
        handle = ctypes.c_void_p()
        _check(_native.load().dk_inmem_index_create(ctypes.byref(d), int(device),
                                                    ctypes.byref(handle)))
        self._handle = handle
        self.dtype = v.dtype
        self.dim = v.shape[1]
        self.capacity = int(capacity)
        self.metric = Metric(int(metric))

    def set_tags(self, first: int, tags) -> None:
        t = np.ascontiguousarray(tags, dtype=np.uint8)
        _check(_native.load().dk_inmem_set_tags(self._handle, int(first), t.size, t.ctypes.data))

    def search(self, params: "Knn", queries):
        """Search a batch of queries of the element type; returns ``(ids, dists, stats)`` with
        external ids (uint64, ``NO_EXTERNAL_ID`` where fewer than k results)."""
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=self.dtype)
        if q.shape[1] != self.dim:
            raise ANNError(Status.DIMENSION_MISMATCH, f"query dim {q.shape[1]} != {self.dim}")
        nq, k = q.shape[0], params.k_value
        ids = np.empty((nq, k), dtype=np.uint64)
        dists = np.empty((nq, k), dtype=np.float32)
        stats = np.zeros(nq, dtype=STATS_DTYPE)
        _check(_native.load().dk_inmem_search(self._handle, q.ctypes.data, q.shape[1], nq, k,
                                              params.l_value, params.beam_width,
                                              ids.ctypes.data, dists.ctypes.data,
                                              stats.ctypes.data))
        return ids, dists, stats

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None:
            _native.load().dk_index_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DiskANNIndex:
    """Graph index over a :class:`GpuProvider`; ``search`` runs batched greedy beam search."""

    def __init__(self, provider: GpuProvider):
        self.provider = provider

    def search(self, params: Knn, strategy: _Strategy, queries, out=None):
        """Search host queries (nq, D) float32; returns ``(ids, distances, stats)`` numpy arrays.

        Host buffers cross the C ABI (``dk_search``): queries are copied to the device and
        results back inside the call.  ``out``: optional caller-owned ``(ids, dists, stats)``
        arrays to write into (uint32 (nq, k), float32 (nq, k), STATS_DTYPE (nq,)), as the
        reference's search writes into the caller's output buffer; pinned host memory makes
        the copies faster.
        """
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        if q.shape[1] != self.provider.dim:
            raise ANNError(Status.DIMENSION_MISMATCH, f"query dim {q.shape[1]} != {self.provider.dim}")
        nq, k = q.shape[0], params.k_value
        if out is not None:
            ids, dists, stats = out
            if (ids.shape != (nq, k) or ids.dtype != np.uint32 or dists.shape != (nq, k)
                    or dists.dtype != np.float32 or stats.shape != (nq,) or stats.dtype != STATS_DTYPE
                    or not all(a.flags["C_CONTIGUOUS"] for a in out)):
                raise ANNError(Status.INVALID_ARGUMENT, "out arrays do not match (nq, k)")
        else:
            ids = np.empty((nq, k), dtype=np.uint32)
            dists = np.empty((nq, k), dtype=np.float32)
            stats = np.zeros(nq, dtype=STATS_DTYPE)
        _check(_native.load().dk_search(
            self.provider.handle, strategy.code, q.ctypes.data, q.shape[1], nq, k,
            params.l_value, params.beam_width, ids.ctypes.data, dists.ctypes.data, stats.ctypes.data,
        ))
        return ids, dists, stats

    def range_search(self, params: Range, queries, capacity: int | None = None):
        """Range search of host queries (FullPrecision, ``dk_range_search``).  Returns
        ``(results, stats)``: per query a ``(ids, dists)`` pair of its results, and the stats
        array (flags bit 1: second round ran; bit 2: results reached the capacity)."""
        ids, dists, stats = self.range_search_arrays(params, queries, capacity)
        return _rows(ids, dists, stats), stats

    def range_search_arrays(self, params: Range, queries, capacity: int | None = None,
                            out=None):
        """:meth:`range_search` returning ``(ids, dists, stats)`` arrays: ``(nq, capacity)``
        rows whose first ``stats["result_count"]`` entries are the results (the rest are
        unspecified).  ``out``: optional caller-owned ``(ids, dists, stats)`` arrays of those
        shapes and types, reused instead of allocating."""
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        if q.shape[1] != self.provider.dim:
            raise ANNError(Status.DIMENSION_MISMATCH, f"query dim {q.shape[1]} != {self.provider.dim}")
        cap = capacity or params.max_returned or self.provider.num_points
        cap = max(cap, params.starting_l, params.max_returned or 0)
        nq = q.shape[0]
        if out is None:
            ids = np.empty((nq, cap), dtype=np.uint32)
            dists = np.empty((nq, cap), dtype=np.float32)
            stats = np.zeros(nq, dtype=STATS_DTYPE)
        else:
            ids, dists, stats = out
            if (ids.shape != (nq, cap) or ids.dtype != np.uint32 or dists.shape != (nq, cap)
                    or dists.dtype != np.float32 or stats.shape != (nq,)
                    or stats.dtype != STATS_DTYPE or not all(
                        a.flags.c_contiguous for a in (ids, dists, stats))):
                raise ANNError(Status.INVALID_ARGUMENT,
                               "out must be contiguous (nq, capacity) uint32 / float32 arrays "
                               "and an (nq,) stats array")
        _check(_native.load().dk_range_search(
            self.provider.handle, q.ctypes.data, q.shape[1], nq, params.starting_l,
            params.beam_width, params.radius,
            float("nan") if params.inner_radius is None else params.inner_radius,
            params.initial_slack, params.range_slack, params.max_returned or 0, cap,
            ids.ctypes.data, dists.ctypes.data, stats.ctypes.data))
        return ids, dists, stats

    def paged_search(self, queries, l_value: int, init_ids=None, queue_capacity: int = 0):
        """Start a paged search for each query (FullPrecision, ``dk_paged_search_create``;
        index.rs:2080-2160 ``paged_search`` / ``paged_search_with_init_ids``).  ``init_ids``:
        None for the start points, or ``(nq, n_init)`` ids.  Returns a :class:`PagedSearch`."""
        return PagedSearch(self, queries, l_value, init_ids, queue_capacity)

    def search_device(self, params: Knn, strategy: _Strategy, queries, ids, dists, stats,
                      stream=None) -> None:
        """Search device-resident queries; outputs go to caller-allocated device buffers.

        ``queries``: CUDA float32 tensor (nq, D); ``ids``: int32 (nq, k) (bit pattern of
        uint32); ``dists``: float32 (nq, k); ``stats``: int32 (nq, 4).  Asynchronous on
        ``stream`` (a torch.cuda.Stream or raw handle; default: torch's current stream).
        """
        import torch

        if stream is None:
            stream = torch.cuda.current_stream(queries.device)
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        nq = queries.shape[0]
        _check(_native.load().dk_search_device(
            self.provider.handle, strategy.code, queries.data_ptr(), queries.stride(0), nq,
            params.k_value, params.l_value, params.beam_width, ids.data_ptr(), dists.data_ptr(),
            stats.data_ptr(), ctypes.c_void_p(handle),
        ))


    def score(self, strategy: _Strategy, queries, ids) -> np.ndarray:
        """Distances each candidate gets from ``strategy``'s traversal scorer
        (``dk_score_candidates``): ``queries`` (nq, D) float32, ``ids`` (nq, m) candidate ids;
        returns (nq, m) float32 (NaN for an id outside the index)."""
        import torch

        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        c = np.ascontiguousarray(np.atleast_2d(ids), dtype=np.uint32)
        if c.shape[0] != q.shape[0]:
            raise ValueError("one candidate row per query")
        dev = torch.device("cuda", self.provider.device)
        dq = torch.from_numpy(q).to(dev)
        dc = torch.from_numpy(c.view(np.int32)).to(dev)
        out = torch.empty(c.shape, dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream(dev)
        _check(_native.load().dk_score_candidates(
            self.provider.handle, strategy.code, dq.data_ptr(), dq.stride(0), q.shape[0],
            dc.data_ptr(), c.shape[1], out.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize(dev)
        return out.cpu().numpy()


def _rows(ids, dists, stats):
    """Per row, the ``(ids, dists)`` of its first ``result_count`` entries."""
    counts = stats["result_count"].tolist()
    return [(ids[i, :c], dists[i, :c]) for i, c in enumerate(counts)]


class PagedSearch:
    """Paged-search sessions, one per query (``dk_paged_search_*``; paged.rs).

    ``next_page(k)`` returns ``(pages, stats)``: per query the ``(ids, dists)`` of its next
    page of at most ``k`` results (empty once its search is exhausted), and the stats array
    (running ``cmps`` / ``hops``; flags bit 2: the session's queue filled).  Raises
    ``ANNError`` (``INVALID_ARGUMENT``) for ``k == 0`` or ``k > l_value`` like the reference.
    """

    def __init__(self, index: "DiskANNIndex", queries, l_value: int, init_ids=None,
                 queue_capacity: int = 0):
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        prov = index.provider
        if q.shape[1] != prov.dim:
            raise ANNError(Status.DIMENSION_MISMATCH, f"query dim {q.shape[1]} != {prov.dim}")
        init = None
        if init_ids is not None:
            init = np.ascontiguousarray(np.atleast_2d(init_ids), dtype=np.uint32)
            if init.shape[0] != q.shape[0]:
                raise ANNError(Status.INVALID_ARGUMENT, "init_ids needs one row per query")
        self._index = index
        self.nq = q.shape[0]
        self.l_value = int(l_value)
        handle = ctypes.c_void_p()
        _check(_native.load().dk_paged_search_create(
            prov.handle, q.ctypes.data, q.shape[1], self.nq, self.l_value,
            None if init is None else init.ctypes.data, 0 if init is None else init.shape[1],
            queue_capacity, ctypes.byref(handle)))
        self._h = handle

    def next_page(self, k: int):
        ids, dists, stats = self.next_page_arrays(k)
        return _rows(ids, dists, stats), stats

    def next_page_arrays(self, k: int):
        """:meth:`next_page` returning ``(ids, dists, stats)`` arrays: ``(nq, k)`` rows whose
        first ``stats["result_count"]`` entries are each session's page."""
        ids = np.empty((self.nq, max(k, 1)), dtype=np.uint32)
        dists = np.empty((self.nq, max(k, 1)), dtype=np.float32)
        stats = np.zeros(self.nq, dtype=STATS_DTYPE)
        _check(_native.load().dk_paged_search_next(self._h, k, ids.ctypes.data,
                                                   dists.ctypes.data, stats.ctypes.data))
        return ids, dists, stats

    def close(self) -> None:
        if getattr(self, "_h", None):
            _native.load().dk_paged_search_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class SearchServer:
    """Continuous-admission serving over a :class:`GpuProvider` (``dk_server_*``).

    ``submit`` queues one request with its own ``k`` and ``L`` (up to ``max_k`` / ``max_l``)
    and returns a ticket; queued requests are launched as soon as one of ``streams`` launch
    contexts is free, overlapping on the device with requests already running.  ``poll``
    returns ``(ids, dists, stats)`` once the request is done, else ``None``.  A submit while
    ``queue_depth`` requests are outstanding raises ``ANNError`` with status ``ADMISSION``.
    """

    def __init__(self, provider: GpuProvider, strategy: _Strategy, max_k: int, max_l: int,
                 beam_width: int = 1, queue_depth: int = 1024, max_slots: int = 0,
                 streams: int = 0, memory_bytes: int = 0):
        L = _native.load()
        cfg = _native.ServerConfig(strategy.code, max_k, max_l, beam_width, queue_depth,
                                   max_slots, streams, 0, memory_bytes)
        handle = ctypes.c_void_p()
        _check(L.dk_server_create(provider.handle, ctypes.byref(cfg), ctypes.byref(handle)))
        self._handle = handle
        self.provider = provider
        self.max_k = int(max_k)

    @property
    def handle(self):
        if self._handle is None:
            raise ANNError(Status.INVALID_ARGUMENT, "server is closed")
        return self._handle

    def submit(self, query, k: int, l_value: int) -> int:
        q = np.ascontiguousarray(np.ravel(query), dtype=np.float32)
        if q.shape[0] != self.provider.dim:
            raise ANNError(Status.DIMENSION_MISMATCH, f"query dim {q.shape[0]} != {self.provider.dim}")
        ticket = ctypes.c_uint64()
        _check(_native.load().dk_server_submit(self.handle, q.ctypes.data, k, l_value,
                                               ctypes.byref(ticket)))
        return int(ticket.value)

    def poll(self, ticket: int, k: int):
        ids = np.empty(k, dtype=np.uint32)
        dists = np.empty(k, dtype=np.float32)
        stats = np.zeros(1, dtype=STATS_DTYPE)
        rc = _native.load().dk_server_poll(self.handle, ticket, ids.ctypes.data,
                                           dists.ctypes.data, stats.ctypes.data)
        if rc == Status.NOT_READY:
            return None
        _check(rc)
        return ids, dists, stats[0]

    def cancel(self, ticket: int) -> None:
        """Cancel an outstanding request (``dk_server_cancel``); its next ``poll`` raises
        ``ANNError`` with status ``CANCELLED``."""
        _check(_native.load().dk_server_cancel(self.handle, ticket))

    def wait(self, ticket: int, k: int, timeout_s: float = 30.0):
        """Poll until the request completes (``TimeoutError`` after ``timeout_s``)."""
        import time

        deadline = time.monotonic() + timeout_s
        while True:
            r = self.poll(ticket, k)
            if r is not None:
                return r
            if time.monotonic() > deadline:
                raise TimeoutError(f"request {ticket} not done after {timeout_s} s")
            time.sleep(0)

    def replay(self, queries, ks, ls, arrival_s, want_results: bool = False):
        """Replay a request stream natively (``dk_server_replay``): request i uses query row
        i % len(queries), ks[i], ls[i] and arrives arrival_s[i] seconds after the start.
        Returns latencies in seconds (and ``(ids, dists)`` with ``want_results``)."""
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=np.float32)
        ks = np.ascontiguousarray(ks, dtype=np.uint32)
        ls = np.ascontiguousarray(ls, dtype=np.uint32)
        arr = np.ascontiguousarray(np.round(np.asarray(arrival_s) * 1e9), dtype=np.uint64)
        n = len(arr)
        lat = np.zeros(n, dtype=np.uint64)
        ids = np.empty((n, self.max_k), np.uint32) if want_results else None
        dists = np.empty((n, self.max_k), np.float32) if want_results else None
        _check(_native.load().dk_server_replay(
            self.handle, q.ctypes.data, q.shape[1], q.shape[0], ks.ctypes.data, ls.ctypes.data,
            arr.ctypes.data, n, lat.ctypes.data, None if ids is None else ids.ctypes.data,
            None if dists is None else dists.ctypes.data))
        lat_s = lat.astype(np.float64) / 1e9
        return (lat_s, ids, dists) if want_results else lat_s

    def info(self) -> dict:
        inf = _native.ServerInfo()
        _check(_native.load().dk_server_get_info(self.handle, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in inf._fields_ if f != "pad"}

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None:
            _native.load().dk_server_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
