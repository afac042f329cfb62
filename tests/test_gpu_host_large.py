"""Host-pointer searches of the batched forms on batches of 8192 queries and
more (results copied back before the status checks, the learned judge's rows
appended to the batch, the device fallback's counters read afterwards): the
answers must be those of one device-pointer search of the whole batch and of
the plain form."""
import numpy as np
import pytest
import torch

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    x, q = datasets.gmm_uint8(120_000, 9_500, d=64, ncomp=1024, sigma=40.0, seed=17)
    idx = hb.Index(64, 128, 16)
    idx.train(x)
    idx.add(x)
    return idx, x, q


def _device_search(idx, q, k):
    dq = torch.from_numpy(q).cuda()
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    idx.search_device(q.shape[0], dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(),
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return dD.cpu().numpy(), dI.cpu().numpy()


@pytest.mark.parametrize("n", [8192, 9_500])
def test_host_search_equals_device_search(big, n):
    idx, x, q = big
    qs = q[:n]
    Dp, Ip = idx.search(qs, 30)
    idx.set_form("bf16")
    try:
        Dh, Ih = idx.search(qs, 30)
        Dd, Id = _device_search(idx, qs, 30)
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(Ih, Id)
    np.testing.assert_array_equal(Dh, Dd)
    np.testing.assert_array_equal(Ih, Ip)
    np.testing.assert_array_equal(Dh, Dp)


def test_fallback_counters_of_a_large_batch(big):
    idx, x, q = big
    Dp, Ip = idx.search(q, 100)
    idx.set_form("bf16")
    idx.set_batch_params(capq=256)
    try:
        Dh, Ih = idx.search(q, 100)
        st = idx.last_stats()
    finally:
        idx.set_batch_params(capq=8192)
        idx.set_form("plain")
    assert st["fallback_queries"] > 0
    np.testing.assert_array_equal(Ih, Ip)
    np.testing.assert_array_equal(Dh, Dp)


def test_learned_judge_rows_of_a_large_batch(big):
    idx, x, q = big
    idx.train_probe_model(q[:4000], max_nprobe=16, k_label=10, epochs=10, lr=1e-3, coverage=0.95)
    idx.set_form("bf16")
    try:
        idx.set_learned(True, judge_fraction=0.0)
        Dd, Id = _device_search(idx, q, 10)
        idx.set_learned(True, judge_fraction=0.01, judge_recall=0.0)
        Dh, Ih = idx.search(q, 10)
        st = idx.last_stats()
    finally:
        idx.set_learned(False)
        idx.set_form("plain")
    assert st["learned_fallback"] == 0
    assert 0.0 < st["judge_recall"] <= 1.0
    np.testing.assert_array_equal(Ih, Id)
    np.testing.assert_array_equal(Dh, Dd)
