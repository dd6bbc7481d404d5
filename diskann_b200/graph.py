"""Graph construction, medoid and PQ tooling over the C ABI (host code in dk_build.cpp)."""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native
from .index import ANNError, Metric, PQData, _check


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


def _lib():
    L = _native.load()
    if not getattr(L, "_dk_build_bound", False):
        u32, u64, i32, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p
        L.dk_distance.restype = i32
        L.dk_distance.argtypes = [i32, vp, vp, u32, vp]
        L.dk_compute_medoid.restype = i32
        L.dk_compute_medoid.argtypes = [vp, u64, u32, u32, vp]
        L.dk_build_vamana.restype = i32
        L.dk_build_vamana.argtypes = [vp, u64, u32, u32, u32, i32, ctypes.POINTER(BuildParams), vp, u64, vp]
        L.dk_build_vamana_device.restype = i32
        L.dk_build_vamana_device.argtypes = [vp, u64, u32, u32, u32, i32, ctypes.POINTER(BuildParams),
                                             vp, u64, vp, i32]
        L.dk_pq_train.restype = i32
        L.dk_pq_train.argtypes = [vp, u64, u32, u32, u32, u32, u64, u32, vp, vp]
        L.dk_pq_encode.restype = i32
        L.dk_pq_encode.argtypes = [vp, u64, u32, u32, u32, vp, vp, u32, vp, u64]
        L._dk_build_bound = True
    return L


def distance(metric: int, x: np.ndarray, y: np.ndarray) -> float:
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    out = ctypes.c_float()
    _check(_lib().dk_distance(int(metric), x.ctypes.data, y.ctypes.data, x.size, ctypes.byref(out)))
    return float(out.value)


def compute_medoid(base: np.ndarray) -> int:
    base = np.ascontiguousarray(base, np.float32)
    out = ctypes.c_uint32()
    _check(_lib().dk_compute_medoid(base.ctypes.data, base.shape[1], base.shape[0], base.shape[1],
                                    ctypes.byref(out)))
    return int(out.value)


def slot_width(pruned_degree: int) -> int:
    """Adjacency slot width used by the reference benchmark: floor(1.3 R)
    (diskann-benchmark/src/inputs/graph_index.rs:690-692)."""
    return int(np.float32(pruned_degree) * np.float32(1.3))


def build_vamana(base: np.ndarray, metric=Metric.L2, pruned_degree: int = 32, l_build: int = 50,
                 alpha: float = 1.2, max_degree: int | None = None, backedge_ratio: float = 1.0,
                 num_threads: int = 0, max_batch: int = 0, device: int | None = None):
    """Build a Vamana graph with one frozen start point (a copy of the medoid row, id N).

    ``device``: search the larger batches on that CUDA device (``dk_build_vamana_device``; the
    same graph, faster).  Returns ``(vectors, adjacency, degrees, n)`` ready for
    :class:`GpuProvider`.
    """
    base = np.ascontiguousarray(base, np.float32)
    n, dim = base.shape
    med = compute_medoid(base)
    vectors = np.vstack([base, base[med : med + 1]])
    md = max_degree or slot_width(pruned_degree)
    adjacency = np.zeros((n + 1, md), np.uint32)
    degrees = np.zeros(n + 1, np.uint32)
    p = BuildParams(pruned_degree, md, l_build, alpha,
                    int(np.ceil(backedge_ratio * pruned_degree)), 0, num_threads, max_batch)
    if device is None:
        _check(_lib().dk_build_vamana(vectors.ctypes.data, dim, n, 1, dim, int(metric),
                                      ctypes.byref(p), adjacency.ctypes.data, md,
                                      degrees.ctypes.data))
    else:
        _check(_lib().dk_build_vamana_device(vectors.ctypes.data, dim, n, 1, dim, int(metric),
                                             ctypes.byref(p), adjacency.ctypes.data, md,
                                             degrees.ctypes.data, int(device)))
    return vectors, adjacency, degrees, n


def train_pq(sample: np.ndarray, chunks: int, iters: int = 12, seed: int = 0, num_threads: int = 0):
    sample = np.ascontiguousarray(sample, np.float32)
    n, dim = sample.shape
    offsets = np.zeros(chunks + 1, np.uint32)
    pivots = np.zeros((256, dim), np.float32)
    _check(_lib().dk_pq_train(sample.ctypes.data, dim, n, dim, chunks, iters, seed, num_threads,
                              offsets.ctypes.data, pivots.ctypes.data))
    return offsets, pivots


def encode_pq(vectors: np.ndarray, offsets: np.ndarray, pivots: np.ndarray, num_threads: int = 0):
    vectors = np.ascontiguousarray(vectors, np.float32)
    n, dim = vectors.shape
    chunks = len(offsets) - 1
    codes = np.zeros((n, chunks), np.uint8)
    off = np.ascontiguousarray(offsets, np.uint32)
    piv = np.ascontiguousarray(pivots, np.float32)
    _check(_lib().dk_pq_encode(vectors.ctypes.data, dim, n, dim, chunks, off.ctypes.data,
                               piv.ctypes.data, num_threads, codes.ctypes.data, chunks))
    return codes


def build_pq(vectors: np.ndarray, chunks: int, train_rows: int, seed: int = 0, iters: int = 12,
             num_threads: int = 0) -> PQData:
    """Train on a seeded sample of ``train_rows`` rows and encode every row of ``vectors``."""
    rng = np.random.default_rng(seed)
    n = vectors.shape[0]
    idx = np.sort(rng.choice(n, size=min(train_rows, n), replace=False))
    offsets, pivots = train_pq(vectors[idx], chunks, iters, seed, num_threads)
    codes = encode_pq(vectors, offsets, pivots, num_threads)
    return PQData(offsets, pivots, codes)
