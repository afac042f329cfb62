"""The e4m3 (FP8) tensor-core form and the wide-dimension query groups.

* The e4m3 tcgen05 path (kind::f8f6f4) against an exact float64 product: the
  f32 accumulation the error bound assumes.
* The e4m3 form re-ranking every candidate its bound admits returns the plain
  form's answer; with the default oversampling (4 x k re-ranked) its recall
  against the exact answer is stated and high on a 420-d mixture.
* The bf16 form at d = 200 (64-query groups) and d = 420 (32-query groups)
  returns the plain form's answer bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import _lib, datasets
from tests.golden import cases
from tests.topk_check import probe_tied_rows

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _e4m3_values(rng, shape):
    # Values exactly representable in e4m3: sign x 2^e x (1 + m/8), e in [-4, 4].
    m = rng.integers(0, 8, shape)
    e = rng.integers(-4, 5, shape)
    s = rng.choice([-1.0, 1.0], shape)
    return (s * np.ldexp(1.0 + m / 8.0, e)).astype(np.float32)


def test_e4m3_tensor_core_tile_accumulates_in_f32():
    rng = np.random.default_rng(0)
    A = _e4m3_values(rng, (128, 256))
    B = _e4m3_values(rng, (128, 256))
    D = np.zeros((128, 128), np.float32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.check(_lib.load().hy_selftest_tcgen05_e4m3(p(A), p(B), p(D)))
    exact = A.astype(np.float64) @ B.astype(np.float64).T
    mag = np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64)).T
    # products of two e4m3 values are exact in f32; f32 accumulation of K = 256
    # of them is off by at most (K + 8) 2^-24 of the sum of magnitudes.
    ratio = np.max(np.abs(D - exact) / mag)
    assert ratio <= (256 + 8) * 2.0 ** -24, ratio


def _index(name, form, **batch):
    c = cases.CASES[name]
    x, q = cases.data(name)
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    idx.centroid_codes = np.load(os.path.join(GOLD, f"{name}.npz"))["centroids"]
    idx.add(x)
    Dp, Ip = idx.search(q, c["k"])
    idx.set_form(form)
    if batch:
        idx.set_batch_params(**batch)
    return idx, x, q, c, Dp, Ip


@pytest.mark.parametrize("name", ["c1", "int_small", "odd_dim", "ip_small", "exhaustive"])
def test_fp8_full_rerank_equals_plain(name):
    """oversample 1000 lets the re-rank take every candidate its error bound
    admits (up to 4096), so the answer is the plain form's."""
    idx, x, q, c, Dp, Ip = _index(name, "fp8", oversample=1000)
    D, I = idx.search(q, c["k"])
    np.testing.assert_array_equal(I, Ip)
    np.testing.assert_array_equal(D, Dp)


@pytest.fixture(scope="module")
def wide():
    x, q = datasets.gmm_dense(60_000, 400, d=420, ncomp=256, sigma=0.3, seed=9)
    idx = hb.Index(420, 128, 16)
    idx.train(x)
    idx.add(x)
    D, I = idx.search(q, 10)
    return idx, x, q, D, I


def test_fp8_oversampled_recall_on_420d(wide):
    idx, x, q, Dp, Ip = wide
    idx.set_form("fp8")
    try:
        D, I = idx.search(q, 10)
        st = idx.last_stats()
    finally:
        idx.set_form("plain")
    recall = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(I.tolist(), Ip.tolist())])
    assert recall >= 0.95, recall
    # every returned distance is the exact FP32 distance of its row
    same = I == Ip
    np.testing.assert_array_equal(D[same], Dp[same])


@pytest.mark.parametrize("d", [200, 420])
def test_bf16_wide_groups_equal_plain(d, wide):
    if d == 420:
        idx, x, q, Dp, Ip = wide
    else:
        x, q = datasets.gmm_dense(40_000, 300, d=200, ncomp=200, sigma=0.3, seed=10)
        idx = hb.Index(200, 100, 12)
        idx.train(x)
        idx.add(x)
        Dp, Ip = idx.search(q, 10)
    idx.set_form("bf16")
    try:
        D, I = idx.search(q, 10)
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(I, Ip)
    np.testing.assert_array_equal(D, Dp)


def test_forms_reject_too_wide():
    idx = hb.Index(2000, 4, 2)
    with pytest.raises(hb.HyError):
        idx.set_form("bf16")
