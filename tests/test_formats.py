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
