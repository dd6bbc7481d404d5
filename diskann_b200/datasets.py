"""Seeded synthetic inputs.

* ``grid``: the reference's lattice workload (diskann/src/graph/test/synthetic.rs:21-348):
  points enumerated with the last coordinate varying fastest, each connected to its axis
  neighbours, plus one frozen start point ``[size] * dim`` whose only neighbour is the last
  point (synthetic.rs:295-348; provider.rs:323-338).
* ``gaussian_mixture`` / ``normalized_gaussian``: the benchmark workloads' vector shapes
  (a seeded Gaussian mixture clipped to [0, 255], or isotropic Gaussian rows normalised to
  unit length); ``normalize_rows`` scales a mixture's rows to unit length in place.
"""

from __future__ import annotations

import itertools

import numpy as np


def grid(dims: int, size: int):
    """Return ``(vectors, adjacency, degrees, num_points)`` for a ``dims``-D lattice.

    Rows ``0..size**dims-1`` are lattice points; row ``size**dims`` is the frozen start point.
    Adjacency lists follow synthetic.rs:173-293: for each axis in order, the ``-1`` neighbour
    then the ``+1`` neighbour.
    """
    n = size ** dims
    coords = np.array(list(itertools.product(range(size), repeat=dims)), dtype=np.float32)
    vectors = np.vstack([coords, np.full((1, dims), float(size), dtype=np.float32)])
    max_degree = 2 * dims
    adjacency = np.zeros((n + 1, max_degree), dtype=np.uint32)
    degrees = np.zeros(n + 1, dtype=np.uint32)
    strides = [size ** (dims - 1 - a) for a in range(dims)]
    for i in range(n):
        c = coords[i].astype(np.int64)
        lst = []
        for a in range(dims):
            if c[a] > 0:
                lst.append(i - strides[a])
            if c[a] < size - 1:
                lst.append(i + strides[a])
        adjacency[i, : len(lst)] = lst
        degrees[i] = len(lst)
    adjacency[n, 0] = n - 1
    degrees[n] = 1
    return vectors, adjacency, degrees, n


def gaussian_mixture(n: int, dim: int, components: int, sigma: float, seed: int,
                     mean_range=(0.0, 100.0), clip=(0.0, 255.0), n_queries: int = 0):
    """Seeded Gaussian mixture: component means U[mean_range]^dim, isotropic ``sigma``,
    values clipped to ``clip``.  Returns ``(base, queries)`` float32 arrays; queries are
    drawn from the same mixture with an independent stream."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(mean_range[0], mean_range[1], size=(components, dim)).astype(np.float32)

    def draw(count, r):
        out = np.empty((count, dim), dtype=np.float32)
        chunk = 1 << 16
        for s in range(0, count, chunk):
            e = min(count, s + chunk)
            comp = r.integers(0, components, size=e - s)
            x = means[comp] + r.standard_normal((e - s, dim), dtype=np.float32) * np.float32(sigma)
            np.clip(x, clip[0], clip[1], out=x)
            out[s:e] = x
        return out

    base = draw(n, np.random.default_rng(seed + 1))
    queries = draw(n_queries, np.random.default_rng(seed + 2)) if n_queries else None
    return base, queries


def normalized_gaussian(n: int, dim: int, seed: int, n_queries: int = 0):
    """Isotropic N(0, 1) rows, L2-normalised.  Returns ``(base, queries)``."""
    def draw(count, r):
        out = np.empty((count, dim), dtype=np.float32)
        chunk = 1 << 15
        for s in range(0, count, chunk):
            e = min(count, s + chunk)
            x = r.standard_normal((e - s, dim), dtype=np.float32)
            x /= np.linalg.norm(x, axis=1, keepdims=True)
            out[s:e] = x
        return out

    base = draw(n, np.random.default_rng(seed + 1))
    queries = draw(n_queries, np.random.default_rng(seed + 2)) if n_queries else None
    return base, queries


def normalize_rows(x: np.ndarray, chunk: int = 1 << 16) -> np.ndarray:
    """Scale every row of the float32 array ``x`` to unit L2 norm, in place, a chunk of rows
    at a time (no full-size temporary).  Returns ``x``."""
    for s in range(0, x.shape[0], chunk):
        blk = x[s:s + chunk]
        blk /= np.linalg.norm(blk, axis=1, keepdims=True)
    return x
