"""GPU: dk_search_device_noalloc, the search entry point that allocates no device memory.

It is meant for callers that cannot allocate while they search, such as a process whose
own caching allocator reserved the GPU's memory up front.  Through the C ABI, two calls in
a row must give the same ids and the same distances (tolerance 0: the search is exact) as
the allocating entry point dk_search_device on the same device buffers, and an index or L
whose scratch would not fit the fixed array is refused with DK_ERR_UNSUPPORTED.

This file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

from diskann_b200 import FullPrecision, GpuProvider, Metric, Status, _native
from tests.helpers import queries_like, random_index

pytestmark = pytest.mark.gpu


def _call(fn, prov, q, k, l, ids, dists, stats):
    return fn(prov.handle, FullPrecision().code, q.data_ptr(), q.stride(0), q.shape[0], k, l, 1,
              ids.data_ptr(), dists.data_ptr(), stats.data_ptr(), ctypes.c_void_p(0))


def test_noalloc_matches_dk_search_device_twice_in_a_row():
    import torch

    lib = _native.load()
    v, a, d, n = random_index(20000, 96, 32, seed=21)
    q_np = queries_like(v[:n], 300, seed=22)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    q = torch.from_numpy(q_np).cuda()
    k, l = 10, 80
    ids0 = torch.empty((300, k), dtype=torch.int32, device="cuda")
    d0 = torch.empty((300, k), dtype=torch.float32, device="cuda")
    s0 = torch.empty((300, 4), dtype=torch.int32, device="cuda")
    assert _call(lib.dk_search_device, prov, q, k, l, ids0, d0, s0) == 0
    torch.cuda.synchronize()
    for _ in range(2):
        ids1 = torch.full_like(ids0, -7)
        d1 = torch.full_like(d0, -7.0)
        s1 = torch.zeros_like(s0)
        assert _call(lib.dk_search_device_noalloc, prov, q, k, l, ids1, d1, s1) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ids1.cpu().numpy(), ids0.cpu().numpy())
        np.testing.assert_allclose(d1.cpu().numpy(), d0.cpu().numpy(), rtol=0, atol=0)
        np.testing.assert_array_equal(s1.cpu().numpy()[:, :3], s0.cpu().numpy()[:, :3])


def test_noalloc_refuses_scratch_beyond_its_array(monkeypatch):
    import torch

    lib = _native.load()
    v, a, d, n = random_index(3000, 64, 16, seed=23)
    prov = GpuProvider(v, a, d, n, Metric.L2)
    q = torch.from_numpy(queries_like(v[:n], 8, seed=24)).cuda()
    ids = torch.empty((8, 10), dtype=torch.int32, device="cuda")
    dists = torch.empty((8, 10), dtype=torch.float32, device="cuda")
    stats = torch.empty((8, 4), dtype=torch.int32, device="cuda")
    # 2^24-slot visited tables (64 MiB per warp) cannot fit the fixed array.
    monkeypatch.setenv("DK_KERNEL", "warp")
    monkeypatch.setenv("DK_GTABLE_LOG2", "24")
    rc = _call(lib.dk_search_device_noalloc, prov, q, 10, 40, ids, dists, stats)
    assert rc == Status.UNSUPPORTED
    st, msg = _native.last_error()
    assert st == Status.UNSUPPORTED and "scratch" in msg
    # nq = 0 only performs the per-device set-up.
    assert lib.dk_search_device_noalloc(prov.handle, FullPrecision().code, None, 64, 0, 10, 40, 1,
                                        None, None, None, ctypes.c_void_p(0)) == 0
