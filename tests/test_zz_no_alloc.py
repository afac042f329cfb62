"""The search entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc while serving (their device
memory belongs to another allocator, or an allocation could synchronise the
device or fail under memory pressure mid-serving): they hand in device
buffers and the library keeps its temporaries in a fixed __device__ array.
This file is collected last on purpose; it must also pass when run alone in a
fresh process.  Results are checked against hy_index_search_preassigned (the
allocating entry point) on two calls in a row, with the tolerance of the
other parity tests (tests/topk_check.py)."""
import ctypes as C
import os

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import _lib
from tests.golden import cases
from tests.topk_check import assert_topk_equal

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _index(name):
    c = cases.CASES[name]
    x, q = cases.data(name)
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    idx.centroid_codes = g["centroids"]
    idx.add(x)
    return idx, q, g["probes"], c


def _noalloc(idx, q, probes, k):
    import torch
    L = _lib.load()
    dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    dp = torch.from_numpy(np.ascontiguousarray(probes, np.int64)).cuda()
    dD = torch.full((q.shape[0], k), -1.0, dtype=torch.float32, device="cuda")
    dI = torch.full((q.shape[0], k), -7, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = L.hy_index_search_preassigned_noalloc(idx._h, q.shape[0], C.c_void_p(dq.data_ptr()), k, probes.shape[1],
                                               C.c_void_p(dp.data_ptr()), C.c_void_p(dD.data_ptr()),
                                               C.c_void_p(dI.data_ptr()), C.c_void_p(s))
    return rc, dD.cpu().numpy(), dI.cpu().numpy()


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small"])
def test_noalloc_matches_allocating_entry_point_twice(name):
    idx, q, probes, c = _index(name)
    D0, I0 = idx.search_preassigned(q, c["k"], probes)
    for _ in range(2):
        rc, D, I = _noalloc(idx, q, probes, c["k"])
        assert rc == _lib.HY_OK, _lib.load().hy_last_error()
        assert_topk_equal(D0, I0, D, I, rtol=1e-5, metric=c["metric"])


def test_noalloc_rejects_batches_beyond_its_scratch():
    idx, q, probes, c = _index("c1")
    # 8000 queries with k = 256 need 8000 * 256 * 8 B = 16 MB of per-query
    # top-k parts, twice the 8 MiB scratch: rejected before any launch.
    big = np.repeat(q, 80, axis=0)
    bigp = np.repeat(probes, 80, axis=0)
    rc, _, _ = _noalloc(idx, big, bigp, 256)
    assert rc == _lib.HY_ERR_ARG
    assert b"scratch" in _lib.load().hy_last_error()


def test_noalloc_rejects_out_of_range_list_ids():
    idx, q, probes, c = _index("c1")
    bad = probes.copy()
    bad[3, 2] = c["nlist"] + 5
    rc, _, _ = _noalloc(idx, q, bad, c["k"])
    assert rc == _lib.HY_ERR_ARG
