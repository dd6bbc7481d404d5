"""CPU: reference file formats round-trip and match their documented byte layout."""

import struct

import numpy as np
import pytest

from diskann_b200 import datasets, formats


def test_bin_roundtrip_and_header(tmp_path):
    x = np.arange(24, dtype=np.float32).reshape(6, 4)
    p = tmp_path / "v.bin"
    formats.write_bin(str(p), x)
    raw = p.read_bytes()
    assert struct.unpack("<II", raw[:8]) == (6, 4)
    assert len(raw) == 8 + x.nbytes
    np.testing.assert_array_equal(formats.read_bin(str(p), np.float32), x)


def test_bin_truncated_is_an_error(tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(struct.pack("<II", 10, 4) + b"\0" * 16)
    with pytest.raises(ValueError):
        formats.read_bin(str(p), np.float32)


def test_graph_roundtrip_and_layout(tmp_path):
    v, a, d, n = datasets.grid(3, 4)
    p = tmp_path / "g"
    size = formats.write_graph(str(p), a, d, start=n, num_start_points=1)
    raw = p.read_bytes()
    assert len(raw) == size
    fsize, md, start, nstart = struct.unpack("<QIIQ", raw[:24])
    assert (fsize, md, start, nstart) == (size, a.shape[1], n, 1)
    assert struct.unpack("<I", raw[24:28])[0] == d[0]
    a2, d2, s2, ns2 = formats.read_graph(str(p))
    np.testing.assert_array_equal(d2, d)
    for i in range(len(d)):
        np.testing.assert_array_equal(a2[i, : d[i]], a[i, : d[i]])
    assert (s2, ns2) == (n, 1)


def test_pq_pivots_roundtrip_with_centroid(tmp_path):
    rng = np.random.default_rng(0)
    piv = rng.standard_normal((256, 12)).astype(np.float32)
    off = np.array([0, 4, 8, 12], np.uint32)
    p = tmp_path / "pivots.bin"
    formats.write_pq_pivots(str(p), piv, off)
    piv2, off2 = formats.read_pq_pivots(str(p))
    np.testing.assert_array_equal(piv2, piv)
    np.testing.assert_array_equal(off2, off)
    cen = rng.standard_normal(12).astype(np.float32)
    formats.write_pq_pivots(str(p), piv, off, centroid=cen)
    piv3, _ = formats.read_pq_pivots(str(p))
    np.testing.assert_allclose(piv3, piv + cen[None, :])
    assert p.stat().st_size > formats.PQ_METADATA_SIZE


def test_pq_codes_roundtrip(tmp_path):
    codes = np.random.default_rng(1).integers(0, 256, size=(50, 16), dtype=np.uint8)
    p = tmp_path / "codes.bin"
    formats.write_pq_codes(str(p), codes)
    np.testing.assert_array_equal(formats.read_pq_codes(str(p)), codes)


@pytest.mark.parametrize("metric", [0, 1, 2, 3])
def test_host_distance_matches_oracle(metric):
    """dk_distance (host tooling, C ABI) reproduces the oracle's rounding sequence bit for bit."""
    from diskann_b200 import graph
    from oracle import oracle as O

    rng = np.random.default_rng(40 + metric)
    for n in (1, 7, 8, 13, 16, 31, 32, 33, 96, 100, 128, 384):
        x = rng.standard_normal(n).astype(np.float32)
        y = rng.standard_normal(n).astype(np.float32)
        if metric == 3:
            x /= np.linalg.norm(x)
            y /= np.linalg.norm(y)
        got = np.float32(graph.distance(metric, x, y))
        ref = np.float32(O.distance(metric, x, y))
        assert got.view(np.uint32) == ref.view(np.uint32), (metric, n, got, ref)


# Byte fixtures assembled here from the reference's documented layouts (independently of
# formats.py): the graph file of diskann-providers/src/storage/bin.rs:320-380 (`save_graph`) and
# the PQ pivot file of diskann-providers/src/storage/pq_storage.rs:80-140 (`write_pivot_data`).

def _graph_fixture():
    """3 nodes + 1 frozen start point; lists [1, 2], [], [0], [2]; configured max degree 4;
    start id 3, one start point."""
    lists = [[1, 2], [], [0], [2]]
    body = b"".join(struct.pack("<I", len(l)) + b"".join(struct.pack("<I", x) for x in l)
                    for l in lists)
    size = 24 + len(body)  # index_size starts at 24 and grows by 4 * (1 + len) per list
    return struct.pack("<Q", size) + struct.pack("<I", 4) + struct.pack("<I", 3) + \
        struct.pack("<Q", 1) + body, lists


def test_graph_file_bytes_match_the_reference_layout(tmp_path):
    want, lists = _graph_fixture()
    adj = np.zeros((4, 4), np.uint32)
    deg = np.array([len(l) for l in lists], np.uint32)
    for i, l in enumerate(lists):
        adj[i, : len(l)] = l
    p = tmp_path / "graph"
    formats.write_graph(str(p), adj, deg, start=3, num_start_points=1, max_degree=4)
    assert p.read_bytes() == want
    q = tmp_path / "graph_fixture"
    q.write_bytes(want)
    a2, d2, start, nstart = formats.read_graph(str(q))
    assert (start, nstart) == (3, 1)
    assert d2.tolist() == [2, 0, 1, 1]
    assert [a2[i, : d2[i]].tolist() for i in range(4)] == lists


def test_graph_file_with_a_wrong_size_or_degree_is_an_error(tmp_path):
    want, _ = _graph_fixture()
    p = tmp_path / "short"
    p.write_bytes(want[:-4])
    with pytest.raises(ValueError):
        formats.read_graph(str(p))
    bad = bytearray(want)
    bad[24:28] = struct.pack("<I", 9)  # node 0 claims 9 neighbours > max degree 4
    bad[0:8] = struct.pack("<Q", len(bad))
    p.write_bytes(bytes(bad))
    with pytest.raises(ValueError):
        formats.read_graph(str(p))


def test_pq_pivot_file_bytes_match_the_reference_layout(tmp_path):
    """Offset table (a .bin column of four u64) at 0, zero padding to the 4096-byte metadata
    region, then the pivots .bin (256 x dim f32), the centroid .bin (dim x 1 f32) and the chunk
    offsets .bin ((M+1) x 1 u32), each written right after the previous."""
    dim, offsets = 6, [0, 2, 4, 6]
    piv = np.arange(256 * dim, dtype=np.float32).reshape(256, dim) / 7
    pivots_bin = struct.pack("<II", 256, dim) + piv.astype("<f4").tobytes()
    centroid_bin = struct.pack("<II", dim, 1) + np.zeros(dim, "<f4").tobytes()
    offsets_bin = struct.pack("<II", 4, 1) + np.array(offsets, "<u4").tobytes()
    c0 = 4096
    c1 = c0 + len(pivots_bin)
    c2 = c1 + len(centroid_bin)
    c3 = c2 + len(offsets_bin)
    table = struct.pack("<II", 4, 1) + struct.pack("<4Q", c0, c1, c2, c3)
    want = table + b"\0" * (4096 - len(table)) + pivots_bin + centroid_bin + offsets_bin
    p = tmp_path / "pivots"
    formats.write_pq_pivots(str(p), piv, np.array(offsets, np.uint32))
    assert p.read_bytes() == want
    q = tmp_path / "pivots_fixture"
    q.write_bytes(want)
    piv2, off2 = formats.read_pq_pivots(str(q))
    np.testing.assert_array_equal(piv2, piv)
    assert off2.tolist() == offsets


# PQ training (dk_pq_train, host code) against the reference's rules
# (diskann-quantization/src/views.rs:254-300 chunking; product/train.rs:22-230 k-means++ seeding
# then Lloyd iterations per chunk).

@pytest.mark.parametrize("dim,chunks", [(128, 32), (100, 32), (384, 48), (7, 3), (96, 96)])
def test_pq_chunk_offsets_follow_the_reference_partition(dim, chunks):
    """The first dim % chunks chunks are one element longer (fill_chunk_offsets)."""
    from diskann_b200 import graph

    x = np.random.default_rng(dim).standard_normal((300, dim)).astype(np.float32)
    offsets, _ = graph.train_pq(x, chunks, iters=1, seed=1)
    want = [0]
    for c in range(chunks):
        want.append(want[-1] + dim // chunks + (1 if c < dim % chunks else 0))
    assert offsets.tolist() == want


def _pq_objective(x, offsets, pivots):
    total = 0.0
    for m in range(len(offsets) - 1):
        s, e = int(offsets[m]), int(offsets[m + 1])
        xs, cs = x[:, s:e].astype(np.float64), pivots[:, s:e].astype(np.float64)
        d = (xs ** 2).sum(1)[:, None] - 2 * xs @ cs.T + (cs ** 2).sum(1)[None, :]
        total += float(np.maximum(d.min(1), 0).sum())
    return total


def test_pq_lloyd_objective_does_not_increase():
    """Same seed, more Lloyd iterations: the quantisation error of the training rows never
    grows, and every code is the nearest pivot of its chunk."""
    from diskann_b200 import graph

    x, _ = datasets.gaussian_mixture(3000, 32, 16, 6.0, seed=4)
    objs = []
    for it in (0, 1, 2, 4, 8):
        off, piv = graph.train_pq(x, 8, iters=it, seed=9)
        objs.append(_pq_objective(x, off, piv))
    assert all(b <= a * (1 + 1e-9) for a, b in zip(objs, objs[1:])), objs
    assert objs[-1] < objs[0]
    codes = graph.encode_pq(x, off, piv)
    for m in range(8):
        s, e = int(off[m]), int(off[m + 1])
        d = ((x[:, None, s:e].astype(np.float64) - piv[None, :, s:e]) ** 2).sum(-1)
        np.testing.assert_array_equal(codes[:, m], d.argmin(1))
