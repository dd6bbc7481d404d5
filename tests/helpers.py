"""Shared test fixtures: seeded random graphs, PQ schemas and index builders."""

from __future__ import annotations

import numpy as np

from diskann_b200 import datasets


def random_graph(n_total: int, degree: int, max_degree: int, seed: int, ragged: bool = True):
    """Random adjacency: each node gets up to ``degree`` distinct neighbours (not itself)."""
    rng = np.random.default_rng(seed)
    adj = np.zeros((n_total, max_degree), dtype=np.uint32)
    deg = np.zeros(n_total, dtype=np.uint32)
    for i in range(n_total):
        d = int(rng.integers(1, degree + 1)) if ragged else degree
        nb = rng.choice(n_total - 1, size=d, replace=False)
        nb[nb >= i] += 1
        adj[i, :d] = nb
        deg[i] = d
    return adj, deg


def random_index(n: int, dim: int, degree: int, seed: int, metric: int = 2, frozen: int = 1,
                 normalize: bool = False, max_degree: int | None = None):
    """Gaussian-mixture vectors (or normalised Gaussian), frozen points = copies of the medoid
    row, random graph.  Returns (vectors, adjacency, degrees, n)."""
    if normalize:
        base, _ = datasets.normalized_gaussian(n, dim, seed)
    else:
        base, _ = datasets.gaussian_mixture(n, dim, 8, 10.0, seed)
    mean = base.astype(np.float64).mean(axis=0).astype(np.float32)
    med = int(np.argmin(((base - mean) ** 2).sum(axis=1)))
    frozen_rows = np.repeat(base[med : med + 1], frozen, axis=0)
    vectors = np.vstack([base, frozen_rows])
    adj, deg = random_graph(n + frozen, degree, max_degree or degree, seed + 7)
    return vectors, adj, deg, n


def simple_pq(vectors: np.ndarray, chunks: int, seed: int):
    """PQ schema with pivots sampled from the data and nearest-pivot codes per chunk."""
    n, dim = vectors.shape
    rng = np.random.default_rng(seed)
    offsets = np.linspace(0, dim, chunks + 1).round().astype(np.uint32)
    pivots = vectors[rng.choice(n, size=256, replace=n < 256)].astype(np.float32).copy()
    pivots += rng.standard_normal(pivots.shape).astype(np.float32) * 0.01
    codes = np.zeros((n, chunks), dtype=np.uint8)
    for m in range(chunks):
        s, e = offsets[m], offsets[m + 1]
        d = ((vectors[:, None, s:e].astype(np.float64) - pivots[None, :, s:e]) ** 2).sum(-1)
        codes[:, m] = np.argmin(d, axis=1)
    return offsets, pivots, codes


def queries_like(vectors: np.ndarray, nq: int, seed: int, normalize: bool = False):
    rng = np.random.default_rng(seed)
    idx = rng.choice(vectors.shape[0], size=nq, replace=False)
    q = vectors[idx] + rng.standard_normal((nq, vectors.shape[1])).astype(np.float32) * 2.0
    if normalize:
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


def inmem_fixture(elem: str, n: int, dim: int, seed: int, metric: int = 2,
                  unreadable: float = 0.1, unmapped: float = 0.05, degree: int = 24):
    """A diskann-inmem store: typed vectors (f32 / f16 / u8 / i8) from the mixture, random
    graph, tags (a fraction of data slots not readable), external ids (a fraction unmapped,
    the frozen slot never).  Returns (typed vectors, f32 values, adjacency, degrees, n, tags,
    external ids)."""
    v, adj, deg, n = random_index(n, dim, degree, seed, metric=metric, max_degree=degree + 7)
    if elem == "f16":
        typed = v.astype(np.float16)
    elif elem == "u8":
        typed = np.clip(np.rint(v), 0, 255).astype(np.uint8)
    elif elem == "i8":
        typed = (np.clip(np.rint(v), 0, 255) - 128).astype(np.int8)
    else:
        typed = v.astype(np.float32)
    values = typed.astype(np.float32)
    rng = np.random.default_rng(seed + 11)
    total = typed.shape[0]
    tags = np.full(total, 254, np.uint8)
    tags[n:] = 255
    bad = rng.random(n) < unreadable
    tags[:n][bad] = rng.choice([0, 1, 2], size=int(bad.sum())).astype(np.uint8)
    ext = (np.arange(total, dtype=np.uint64) * 10 + 1).astype(np.uint64)
    ext[n:] = np.uint64(0xFFFFFFFFFFFFFFFF)
    ext[:n][rng.random(n) < unmapped] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return typed, values, adj, deg, n, tags, ext
