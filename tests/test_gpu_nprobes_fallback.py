"""Per-query nprobe and the bf16 form's exact fallback.

* search_nprobes (host and device pointers) returns what a preassigned search
  over each query's first nprobes[i] lists returns, in both forms.
* Queries whose bf16 candidate buffers overflow are answered again by the
  plain scan on the device (device-pointer search included), however many
  of a batch's queries overflow.
"""
import numpy as np
import pytest
import torch

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def skewed():
    # 64 lists over a 512-component mixture; 1,000 queries.
    x, q = datasets.gmm_uint8(40_000, 1_000, d=64, ncomp=512, sigma=30.0, seed=21)
    idx = hb.Index(64, 64, 32)
    idx.train(x)
    idx.add(x)
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=20)
    return idx, x, q


def _cut(probes, npq):
    out = probes.copy()
    for i, n in enumerate(npq):
        out[i, n:] = -1
    return out


@pytest.mark.parametrize("form", ["plain", "bf16"])
def test_search_nprobes_equals_cut_preassigned(skewed, form):
    idx, x, q = skewed
    rng = np.random.default_rng(5)
    npq = rng.integers(1, 33, q.shape[0]).astype(np.int32)
    idx.set_form(form)
    try:
        D, I = idx.search_nprobes(q, 20, npq)
        st = idx.last_stats()
        idx.set_form("plain")
        P = idx.probes(q)
        Dr, Ir = idx.search_preassigned(q, 20, _cut(P, npq))
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(I, Ir)
    np.testing.assert_array_equal(D, Dr)
    assert abs(st["mean_nprobe"] - npq.mean()) < 1e-9


def test_search_nprobes_device_matches_host(skewed):
    idx, x, q = skewed
    rng = np.random.default_rng(6)
    npq = rng.integers(8, 33, q.shape[0]).astype(np.int32)
    idx.set_form("bf16")
    try:
        Dh, Ih = idx.search_nprobes(q, 10, npq)
        dq = torch.from_numpy(q).cuda()
        dn = torch.from_numpy(npq).cuda()
        dD = torch.empty((q.shape[0], 10), dtype=torch.float32, device="cuda")
        dI = torch.empty((q.shape[0], 10), dtype=torch.int64, device="cuda")
        idx.search_nprobes_device(q.shape[0], dq.data_ptr(), 10, dn.data_ptr(), int(npq.max()), dD.data_ptr(),
                                  dI.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(dI.cpu().numpy(), Ih)
    np.testing.assert_array_equal(dD.cpu().numpy(), Dh)


def test_search_nprobes_rejects_zero(skewed):
    idx, x, q = skewed
    with pytest.raises(hb.HyError):
        idx.search_nprobes(q[:4], 10, np.array([1, 0, 2, 3], np.int32))


def test_device_fallback_answers_overflowed_queries_exactly(skewed):
    """capq 256 < the candidates of most queries: the device-pointer search
    answers them with the plain scan on the device."""
    idx, x, q = skewed
    qs = q[:200]
    Dp, Ip = idx.search(qs, 100)
    idx.set_form("bf16")
    idx.set_batch_params(capq=256)
    try:
        dq = torch.from_numpy(qs).cuda()
        dD = torch.empty((qs.shape[0], 100), dtype=torch.float32, device="cuda")
        dI = torch.empty((qs.shape[0], 100), dtype=torch.int64, device="cuda")
        idx.search_device(qs.shape[0], dq.data_ptr(), 100, dD.data_ptr(), dI.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        st = idx.last_stats()
    finally:
        idx.set_batch_params(capq=8192)
        idx.set_form("plain")
    assert st["fallback_queries"] > 0
    np.testing.assert_array_equal(dI.cpu().numpy(), Ip)
    np.testing.assert_array_equal(dD.cpu().numpy(), Dp)


def test_device_fallback_has_no_cap(skewed):
    """All 1,000 queries overflow capq 256 (far more than one wave of the
    fallback's query slots, 148): the device-pointer search answers every
    one exactly with the plain scan on the device, and so does the
    host-pointer search."""
    idx, x, q = skewed
    Dp, Ip = idx.search(q, 100)
    idx.set_form("bf16")
    idx.set_batch_params(capq=256)
    try:
        dq = torch.from_numpy(q).cuda()
        dD = torch.empty((q.shape[0], 100), dtype=torch.float32, device="cuda")
        dI = torch.empty((q.shape[0], 100), dtype=torch.int64, device="cuda")
        idx.search_device(q.shape[0], dq.data_ptr(), 100, dD.data_ptr(), dI.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        st_dev = idx.last_stats()
        D, I = idx.search(q, 100)
        st = idx.last_stats()
    finally:
        idx.set_batch_params(capq=8192)
        idx.set_form("plain")
    assert st_dev["fallback_queries"] > 296
    assert st["fallback_queries"] == st_dev["fallback_queries"]
    np.testing.assert_array_equal(dI.cpu().numpy(), Ip)
    np.testing.assert_array_equal(dD.cpu().numpy(), Dp)
    np.testing.assert_array_equal(I, Ip)
    np.testing.assert_array_equal(D, Dp)
