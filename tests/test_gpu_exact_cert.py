"""The bf16 form's exactness certificate: when the arena and a query hold
integers of magnitude <= 256 with |x|^2 + |q|^2 < 2^23, every product and
partial sum of the tensor-core distance is an integer below 2^24, so the
distance is the plain scan's bit for bit and the re-rank keeps it instead of
recomputing it.  Each case checks the bf16 answer against the plain form's,
on both sides of every condition of the certificate."""
import numpy as np
import pytest

import harmonyclient_b200 as hb

pytestmark = pytest.mark.gpu


def _index(x, nlist=32, nprobe=8):
    idx = hb.Index(x.shape[1], nlist, nprobe)
    idx.train(x)
    idx.add(x)
    return idx


def _both(idx, q, k):
    Dp, Ip = idx.search(q, k)
    idx.set_form("bf16")
    try:
        Db, Ib = idx.search(q, k)
    finally:
        idx.set_form("plain")
    return Dp, Ip, Db, Ib


def _mixture(rng, n, d, hi, ncomp=64, sigma=12.0):
    c = rng.uniform(0, hi, (ncomp, d))
    lab = rng.integers(0, ncomp, n)
    return np.clip(np.rint(c[lab] + rng.normal(0, sigma, (n, d))), 0, hi).astype(np.float32)


@pytest.mark.parametrize("k", [1, 10, 100])
def test_uint8_data_and_queries(k):
    rng = np.random.default_rng(1)
    x = _mixture(rng, 30_000, 128, 255)
    q = _mixture(rng, 500, 128, 255)
    Dp, Ip, Db, Ib = _both(_index(x), q, k)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)


def test_mixed_batch_of_integral_and_fractional_queries():
    rng = np.random.default_rng(2)
    x = _mixture(rng, 20_000, 96, 255)
    q = _mixture(rng, 400, 96, 255)
    q[::3] += 0.5  # a third of the queries are not integral
    q[1::7, 5] = -3.25
    Dp, Ip, Db, Ib = _both(_index(x), q, 20)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)


def test_norms_at_the_certificate_limit():
    """Values near 256 in 128 dimensions: |x|^2 + |q|^2 crosses 2^23 for
    some pairs, which then take the recomputed path."""
    rng = np.random.default_rng(3)
    x = _mixture(rng, 20_000, 128, 256, sigma=3.0)
    x[:5000] = np.clip(x[:5000] + 200, 0, 256)
    q = np.concatenate([x[rng.integers(0, 20_000, 200)], _mixture(rng, 200, 128, 256, sigma=3.0)])
    assert (np.sum(x.astype(np.float64) ** 2, 1).max() + np.sum(q.astype(np.float64) ** 2, 1).max()) > 2 ** 23
    Dp, Ip, Db, Ib = _both(_index(x), q, 50)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)


def test_integers_beyond_bf16_precision():
    """Integers up to 600 are not all exact in bf16: no certificate."""
    rng = np.random.default_rng(4)
    x = _mixture(rng, 20_000, 64, 600, sigma=20.0)
    q = _mixture(rng, 300, 64, 600, sigma=20.0)
    Dp, Ip, Db, Ib = _both(_index(x), q, 10)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)


def test_signed_integers_inner_product():
    rng = np.random.default_rng(5)
    x = np.rint(rng.normal(0, 20, (20_000, 64))).clip(-128, 127).astype(np.float32)
    q = np.rint(rng.normal(0, 20, (300, 64))).clip(-128, 127).astype(np.float32)
    idx = hb.Index(64, 32, 8, 0)
    idx.train(x)
    idx.add(x)
    Dp, Ip, Db, Ib = _both(idx, q, 10)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)
