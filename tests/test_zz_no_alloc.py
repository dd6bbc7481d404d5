"""GPU: dk_search_device_noalloc, the search entry point that allocates no device memory.

It is meant for callers that cannot allocate while they search, such as a process whose
own caching allocator reserved the GPU's memory up front.  Through the C ABI, two calls in
a row must give the same ids, distances (tolerance 0: the search is exact) and statistics as
the allocating entry point dk_search_device on the same device buffers, and as the oracle.
That holds on the warp-per-query path (beam 1), on the CTA-per-query path (beam 8, whose
tables and spill bitmaps are laid out differently in the fixed array), and when the visited
sets are forced into the spill pass, whose bitmaps then come from the fixed array too.  An
index or L whose scratch would not fit the fixed array is refused with DK_ERR_UNSUPPORTED.

This file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

from diskann_b200 import FullPrecision, GpuProvider, Metric, Status, _native
from oracle import oracle as O
from tests.helpers import queries_like, random_index

pytestmark = pytest.mark.gpu


def _call(fn, prov, q, k, l, beam, ids, dists, stats):
    return fn(prov.handle, FullPrecision().code, q.data_ptr(), q.stride(0), q.shape[0], k, l, beam,
              ids.data_ptr(), dists.data_ptr(), stats.data_ptr(), ctypes.c_void_p(0))


def _outputs(nq, k, device_fill):
    import torch

    ids = torch.full((nq, k), device_fill, dtype=torch.int32, device="cuda")
    dists = torch.full((nq, k), float(device_fill), dtype=torch.float32, device="cuda")
    stats = torch.zeros((nq, 4), dtype=torch.int32, device="cuda")
    return ids, dists, stats


def _check_against(prov, orc, q_np, k, l, beam):
    """dk_search_device once, then dk_search_device_noalloc twice; all three equal each other
    and the oracle bit for bit (ids, float32 distance bits, cmps, hops, result_count)."""
    import torch

    lib = _native.load()
    nq = q_np.shape[0]
    q = torch.from_numpy(q_np).cuda()
    ids0, d0, s0 = _outputs(nq, k, -7)
    assert _call(lib.dk_search_device, prov, q, k, l, beam, ids0, d0, s0) == 0
    torch.cuda.synchronize()
    oi, od, ost = orc.search(q_np, k, l, beam, O.STRATEGY_FULL_PRECISION, threads=4)
    ref_ids = ids0.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(ref_ids, oi)
    np.testing.assert_array_equal(d0.cpu().numpy().view(np.uint32), od.view(np.uint32))
    flags = []
    for _ in range(2):
        ids1, d1, s1 = _outputs(nq, k, -7)
        assert _call(lib.dk_search_device_noalloc, prov, q, k, l, beam, ids1, d1, s1) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ids1.cpu().numpy(), ids0.cpu().numpy())
        np.testing.assert_allclose(d1.cpu().numpy(), d0.cpu().numpy(), rtol=0, atol=0)
        s = s1.cpu().numpy()
        np.testing.assert_array_equal(s[:, :3], s0.cpu().numpy()[:, :3])
        np.testing.assert_array_equal(s[:, 0].astype(np.uint32), ost["cmps"])
        np.testing.assert_array_equal(s[:, 1].astype(np.uint32), ost["hops"])
        np.testing.assert_array_equal(s[:, 2].astype(np.uint32), ost["result_count"])
        flags.append(s[:, 3])
    return flags


@pytest.mark.parametrize("path,beam", [("warp", 1), ("cta", 8)])
def test_noalloc_matches_dk_search_device_and_oracle_twice_in_a_row(path, beam, monkeypatch):
    monkeypatch.setenv("DK_KERNEL", path)
    v, a, d, n = random_index(20000, 96, 32, seed=21)
    q_np = queries_like(v[:n], 300, seed=22)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    _check_against(prov, orc, q_np, 10, 80, beam)


@pytest.mark.parametrize("path,beam", [("warp", 1), ("cta", 8)])
def test_noalloc_spill_pass_from_the_fixed_array(path, beam, monkeypatch):
    """Visited levels far too small for L = 200: queries spill, and the bitmap pass runs with
    its bitmaps carved from the fixed array; results stay exact."""
    monkeypatch.setenv("DK_KERNEL", path)
    v, a, d, n = random_index(4000, 32, 30, seed=31, max_degree=30)
    q_np = queries_like(v[:n], 40, seed=32)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    orc = O.OracleIndex(v, a, d, n, O.METRIC_L2)
    monkeypatch.setenv("DK_HASH_LOG2", "8")
    monkeypatch.setenv("DK_GTABLE_LOG2", "8")
    flags = _check_against(prov, orc, q_np, 10, 200, beam)
    assert all((f & 1).any() for f in flags)


def test_noalloc_refuses_scratch_beyond_its_array(monkeypatch):
    import torch

    lib = _native.load()
    v, a, d, n = random_index(3000, 64, 16, seed=23)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    q = torch.from_numpy(queries_like(v[:n], 8, seed=24)).cuda()
    ids, dists, stats = _outputs(8, 10, 0)
    # 2^24-slot visited tables (64 MiB per warp) cannot fit the fixed array.
    monkeypatch.setenv("DK_KERNEL", "warp")
    monkeypatch.setenv("DK_GTABLE_LOG2", "24")
    rc = _call(lib.dk_search_device_noalloc, prov, q, 10, 40, 1, ids, dists, stats)
    assert rc == Status.UNSUPPORTED
    st, msg = _native.last_error()
    assert st == Status.UNSUPPORTED and "scratch" in msg
    # nq = 0 only performs the per-device set-up.
    assert lib.dk_search_device_noalloc(prov.handle, FullPrecision().code, None, 64, 0, 10, 40, 1,
                                        None, None, None, ctypes.c_void_p(0)) == 0
