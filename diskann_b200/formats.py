"""The reference's on-disk formats, so an index built by the reference loads here and back.

* ``.bin`` matrices (diskann-utils/src/io.rs:24-60; storage/bin.rs:131-175): little-endian
  ``u32 npoints, u32 ndims`` then the rows densely in their native element type.
* Graph files (diskann-providers/src/storage/bin.rs:234-340): a 24-byte header
  (``u64 file_size, u32 max_degree, u32 start, u64 num_start_points``) followed, for every
  node in id order, by ``u32 len`` and ``len`` u32 neighbour ids.
* PQ pivots (diskann-providers/src/storage/pq_storage.rs:92-130, 278-348): a 4096-byte
  metadata region holding a ``.bin`` of four u64 file offsets; at those offsets a ``.bin``
  of the pivots (256 x dim f32), of the centroid (dim x 1 f32; added back to the pivots on
  load when non-zero) and of the chunk offsets ((M+1) x 1 u32).
* PQ codes: a ``.bin`` of u8 (npoints x M).
"""

from __future__ import annotations

import struct

import numpy as np

PQ_METADATA_SIZE = 4096


def write_bin(path: str, data: np.ndarray) -> int:
    data = np.ascontiguousarray(data)
    if data.ndim == 1:
        data = data.reshape(-1, 1)
    with open(path, "wb") as f:
        f.write(struct.pack("<II", data.shape[0], data.shape[1]))
        f.write(data.tobytes())
    return 8 + data.nbytes


def _bin_bytes(data: np.ndarray) -> bytes:
    data = np.ascontiguousarray(data)
    if data.ndim == 1:
        data = data.reshape(-1, 1)
    return struct.pack("<II", data.shape[0], data.shape[1]) + data.tobytes()


def read_bin(path: str, dtype, offset: int = 0) -> np.ndarray:
    with open(path, "rb") as f:
        f.seek(offset)
        npts, ndims = struct.unpack("<II", f.read(8))
        count = npts * ndims
        data = np.frombuffer(f.read(count * np.dtype(dtype).itemsize), dtype=dtype)
    if data.size != count:
        raise ValueError(f"{path}: expected {count} elements after the header, found {data.size}")
    return data.reshape(npts, ndims).copy()


def write_graph(path: str, adjacency: np.ndarray, degrees: np.ndarray, start: int,
                num_start_points: int, max_degree: int | None = None) -> int:
    """Write every row (frozen points included) in id order; returns the file size."""
    degrees = np.asarray(degrees, dtype=np.uint32)
    body = bytearray()
    for i in range(adjacency.shape[0]):
        d = int(degrees[i])
        body += struct.pack("<I", d)
        body += np.ascontiguousarray(adjacency[i, :d], dtype="<u4").tobytes()
    size = 24 + len(body)
    md = int(max_degree if max_degree is not None else adjacency.shape[1])
    with open(path, "wb") as f:
        f.write(struct.pack("<QIIQ", size, md, int(start), int(num_start_points)))
        f.write(body)
    return size


def read_graph(path: str):
    """Return ``(adjacency (n, max_degree) u32, degrees (n,) u32, start, num_start_points)``."""
    with open(path, "rb") as f:
        raw = f.read()
    size, max_degree, start, nstart = struct.unpack_from("<QIIQ", raw, 0)
    if size != len(raw):
        raise ValueError(f"{path}: header says {size} bytes, file has {len(raw)}")
    words = np.frombuffer(raw, dtype="<u4", offset=24)
    rows, degs = [], []
    pos = 0
    while pos < words.size:
        d = int(words[pos])
        if d > max_degree:
            raise ValueError(f"{path}: node {len(degs)} has {d} neighbours > max_degree {max_degree}")
        rows.append(words[pos + 1: pos + 1 + d])
        degs.append(d)
        pos += 1 + d
    adjacency = np.zeros((len(rows), max(1, max_degree)), np.uint32)
    for i, r in enumerate(rows):
        adjacency[i, : r.size] = r
    return adjacency, np.array(degs, np.uint32), int(start), int(nstart)


def write_pq_pivots(path: str, pivots: np.ndarray, offsets: np.ndarray,
                    centroid: np.ndarray | None = None) -> None:
    pivots = np.ascontiguousarray(pivots, np.float32)
    dim = pivots.shape[1]
    centroid = np.zeros(dim, np.float32) if centroid is None else np.asarray(centroid, np.float32)
    parts = [_bin_bytes(pivots), _bin_bytes(centroid.reshape(dim, 1)),
             _bin_bytes(np.asarray(offsets, np.uint32).reshape(-1, 1))]
    cumul = [PQ_METADATA_SIZE]
    for p in parts:
        cumul.append(cumul[-1] + len(p))
    with open(path, "wb") as f:
        f.write(_bin_bytes(np.array(cumul, np.uint64).reshape(4, 1)))
        f.seek(PQ_METADATA_SIZE)
        for p in parts:
            f.write(p)


def read_pq_pivots(path: str):
    """Return ``(pivots (256, dim) f32, offsets (M+1,) u32)``; a non-zero centroid is added to
    the pivots as the reference's loader does."""
    off = read_bin(path, np.uint64, 0).reshape(-1)
    if off.size != 4:
        raise ValueError(f"{path}: expected 4 offsets, found {off.size}")
    pivots = read_bin(path, np.float32, int(off[0]))
    centroid = read_bin(path, np.float32, int(off[1])).reshape(-1)
    offsets = read_bin(path, np.uint32, int(off[2])).reshape(-1)
    if centroid.size != pivots.shape[1]:
        raise ValueError(f"{path}: centroid has {centroid.size} entries, pivots have dim {pivots.shape[1]}")
    if np.any(centroid != 0):
        pivots = pivots + centroid[None, :]
    return pivots.astype(np.float32), offsets


def write_pq_codes(path: str, codes: np.ndarray) -> None:
    write_bin(path, np.ascontiguousarray(codes, np.uint8))


def read_pq_codes(path: str) -> np.ndarray:
    return read_bin(path, np.uint8)
