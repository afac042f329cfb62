"""The batched bf16 tensor-core form: list-major scan on tcgen05 with an exact
FP32 re-rank.  On integer-valued data in [0,255] its bf16 distances are exact,
so results must equal the reference's bit for bit (up to ties at the k-th
distance); on float data the re-rank restores exact FP32 distances."""
import os

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets
from oracle import port
from tests.golden import cases
from tests.topk_check import assert_topk_equal, probe_tied_rows

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, f"{name}.npz"))


def bf16_index(name, **batch):
    c = cases.CASES[name]
    x, q = cases.data(name)
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    idx.centroid_codes = load(name)["centroids"]
    idx.add(x)
    idx.set_form("bf16")
    if batch:
        idx.set_batch_params(**batch)
    return idx, x, q, c


@pytest.mark.parametrize("name", ["int_small", "c1", "ip_small", "exhaustive", "odd_dim"])
def test_bf16_matches_reference(name):
    idx, x, q, c = bf16_index(name)
    g = load(name)
    D, I = idx.search(q, c["k"])
    tied = probe_tied_rows(q, g["centroids"], g["probes"], c["metric"])
    rtol = 0.0 if name == "int_small" else 1e-5
    assert_topk_equal(g["D"], g["I"], D, I, rtol=rtol, metric=c["metric"], skip_rows=tied)
    assert idx.last_stats()["fallback_queries"] == 0


@pytest.mark.parametrize("name", ["int_small", "c1", "odd_dim", "ip_small", "exhaustive"])
def test_bf16_equals_plain_bit_exact(name):
    """The re-rank set is chosen with rigorous bf16 error bounds, so the bf16
    form returns exactly the plain form's answer on any data."""
    idx, x, q, c = bf16_index(name)
    Db, Ib = idx.search(q, c["k"])
    idx.set_form("plain")
    Dp, Ip = idx.search(q, c["k"])
    np.testing.assert_array_equal(Db, Dp)
    np.testing.assert_array_equal(Ib, Ip)


def test_bf16_overflow_falls_back_to_plain():
    idx, x, q, c = bf16_index("c1", capq=64)
    g = load("c1")
    D, I = idx.search(q, c["k"])
    st = idx.last_stats()
    assert st["fallback_queries"] > 0
    tied = probe_tied_rows(q, g["centroids"], g["probes"])
    assert_topk_equal(g["D"], g["I"], D, I, rtol=1e-5, skip_rows=tied)


def test_bf16_row_slices_and_small_groups():
    """Short row slices split every list into several work items."""
    idx, x, q, c = bf16_index("int_small", row_slice=128)
    g = load("int_small")
    D, I = idx.search(q[:37], c["k"])
    tied = probe_tied_rows(q[:37], g["centroids"], g["probes"][:37])
    assert_topk_equal(g["D"][:37], g["I"][:37], D, I, rtol=0.0, skip_rows=tied)


def test_bf16_device_api_matches_host_api():
    import torch
    idx, x, q, c = bf16_index("int_small")
    Dh, Ih = idx.search(q, c["k"])
    dq = torch.from_numpy(q).cuda()
    dD = torch.empty((q.shape[0], c["k"]), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], c["k"]), dtype=torch.int64, device="cuda")
    idx.search_device(q.shape[0], dq.data_ptr(), c["k"], dD.data_ptr(), dI.data_ptr(),
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dD.cpu().numpy(), Dh)
    np.testing.assert_array_equal(dI.cpu().numpy(), Ih)


@pytest.mark.parametrize("name", ["int_small", "ip_small"])
@pytest.mark.parametrize("k", [1, 32, 33, 100, 129, 256])
def test_bf16_equals_plain_across_k(name, k):
    """The first pass's k-th bound (per-lane register selection, sized by k)
    is valid at every k: the bf16 answer equals the plain scan's."""
    idx, x, q, c = bf16_index(name)
    Db, Ib = idx.search(q, k)
    assert idx.last_stats()["fallback_queries"] == 0
    idx.set_form("plain")
    Dp, Ip = idx.search(q, k)
    np.testing.assert_array_equal(Db, Dp)
    np.testing.assert_array_equal(Ib, Ip)


def test_bf16_equals_plain_duplicated_rows():
    """1,500 copies of one row in a first-pass list, queries next to it:
    the dense tightening's k-th bound falls on a run of equal scores, and the
    answer, ties to the lower id, is still the plain scan's."""
    x, q = datasets.gmm_uint8(20_000, 60, d=32, ncomp=40, seed=3)
    x[:1500] = x[0]
    q[:20] = np.clip(x[0] + np.arange(20)[:, None] % 3, 0, 255)
    idx = hb.Index(32, 8, 1)
    idx.train(x)
    idx.add(x)
    idx.set_form("bf16")
    Db, Ib = idx.search(q, 100)
    idx.set_form("plain")
    Dp, Ip = idx.search(q, 100)
    np.testing.assert_array_equal(Db, Dp)
    np.testing.assert_array_equal(Ib, Ip)


def test_bf16_equals_plain_long_dense_lists():
    """First-pass lists of about 5,000 rows (dense tightening over many
    rounds of 128 scores per warp): the answer is still the plain scan's."""
    x, q = datasets.gmm_uint8(60_000, 300, d=32, ncomp=40, seed=7)
    idx = hb.Index(32, 12, 2)
    idx.train(x)
    idx.add(x)
    idx.set_form("bf16")
    Db, Ib = idx.search(q, 100)
    idx.set_form("plain")
    Dp, Ip = idx.search(q, 100)
    np.testing.assert_array_equal(Db, Dp)
    np.testing.assert_array_equal(Ib, Ip)


@pytest.mark.parametrize("qg", [32, 64, 128])
def test_bf16_group_sizes_equal_plain(qg):
    """Every query-group size (and with it the copy-ring depth) returns the
    plain scan's answer; groups smaller than a list's query count split it."""
    idx, x, q, c = bf16_index("int_small")
    idx.set_group_size(qg)
    Db, Ib = idx.search(q, c["k"])
    assert idx.last_stats()["fallback_queries"] == 0
    idx.set_form("plain")
    Dp, Ip = idx.search(q, c["k"])
    np.testing.assert_array_equal(Db, Dp)
    np.testing.assert_array_equal(Ib, Ip)
