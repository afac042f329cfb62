"""The bf16 form's coarse step on the tensor cores: bf16 scores of every
centroid with error bounds, exact FP32 scores only for the centroids whose
bound can reach the nprobe best.  Its probe lists must equal the exact
coarse step's (every centroid scored in FP32, then the nprobe best with ties
to the lower centroid), and so must the searches built on them."""
import os

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets
from tests.golden import cases

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(name):
    c = cases.CASES[name]
    x, q = cases.data(name)
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    idx.centroid_codes = np.load(os.path.join(GOLD, f"{name}.npz"))["centroids"]
    idx.add(x)
    return idx, x, q, c


def _probes(idx, q, mode):
    idx.set_form("bf16")
    idx.set_coarse(mode)
    try:
        return idx.probes(q)
    finally:
        idx.set_coarse("tensor")
        idx.set_form("plain")


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small", "exhaustive", "odd_dim"])
def test_tensor_probes_equal_exact(name):
    idx, x, q, c = _golden(name)
    plain = idx.probes(q)
    np.testing.assert_array_equal(_probes(idx, q, "exact"), plain)
    np.testing.assert_array_equal(_probes(idx, q, "tensor"), plain)


@pytest.mark.parametrize("d", [4, 8, 12, 20, 36])
def test_tensor_probes_equal_exact_small_dims(d):
    """The exact re-scoring stages centroid rows in two dimension halves (at
    d = 4 the second half is empty); 70 probes of 300 lists take three
    rounds of 32 rows."""
    x, q = datasets.gmm_float(20_000, 400, d=d, ncomp=300, seed=50 + d)
    idx = hb.Index(d, 300, 70)
    idx.train(x)
    idx.add(x)
    plain = idx.probes(q)
    np.testing.assert_array_equal(_probes(idx, q, "tensor"), plain)
    idx.set_form("bf16")
    try:
        Dt, It = idx.search(q, 10)
    finally:
        idx.set_form("plain")
    Dp, Ip = idx.search(q, 10)
    np.testing.assert_array_equal(It, Ip)
    np.testing.assert_array_equal(Dt, Dp)


@pytest.fixture(scope="module")
def wide():
    # 1,000 lists (not a multiple of 128), 3,000 queries, integer data.
    x, q = datasets.gmm_uint8(100_000, 3_000, d=128, ncomp=2_000, sigma=20.0, seed=41)
    idx = hb.Index(128, 1000, 64)
    idx.train(x)
    idx.add(x)
    return idx, x, q


@pytest.mark.parametrize("nprobe", [1, 17, 64, 256])
def test_tensor_probes_equal_exact_many_lists(wide, nprobe):
    idx, x, q = wide
    idx.nprobe = nprobe
    try:
        plain = idx.probes(q)
        got = _probes(idx, q, "tensor")
    finally:
        idx.nprobe = 64
    np.testing.assert_array_equal(got, plain)


def test_tensor_probes_with_duplicate_centroids(wide):
    """Equal scores from duplicated centroids: ties go to the lower centroid."""
    idx, x, q = wide
    cent = idx.centroid_codes.copy()
    other = hb.Index(128, 1000, 32)
    cent[500:510] = cent[0:10]
    other.centroid_codes = cent
    other.add(x[:20_000])
    plain = other.probes(q[:500])
    np.testing.assert_array_equal(_probes(other, q[:500], "tensor"), plain)


def test_search_same_with_either_coarse_step(wide):
    idx, x, q = wide
    idx.set_form("bf16")
    try:
        idx.set_coarse("exact")
        De, Ie = idx.search(q, 50)
        idx.set_coarse("tensor")
        Dt, It = idx.search(q, 50)
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(It, Ie)
    np.testing.assert_array_equal(Dt, De)


def test_set_coarse_rejects_unknown_mode(wide):
    idx, x, q = wide
    with pytest.raises(hb.HyError):
        idx.set_coarse(7)


@pytest.fixture(scope="module")
def many_lists():
    # 4,096 lists (above 2,048: the two-launch tensor-core coarse step).
    x, q = datasets.gmm_uint8(200_000, 2_000, d=64, ncomp=4_096, sigma=15.0, seed=43)
    idx = hb.Index(64, 4096, 64)
    idx.train(x)
    idx.add(x)
    return idx, x, q


@pytest.mark.parametrize("nprobe", [1, 32, 128, 256])
def test_tensor_probes_equal_exact_above_2048_lists(many_lists, nprobe):
    idx, x, q = many_lists
    idx.nprobe = nprobe
    try:
        plain = idx.probes(q)
        got = _probes(idx, q, "tensor")
    finally:
        idx.nprobe = 64
    np.testing.assert_array_equal(got, plain)


def test_search_above_2048_lists_equals_plain(many_lists):
    idx, x, q = many_lists
    Dp, Ip = idx.search(q, 20)
    idx.set_form("bf16")
    try:
        Dt, It = idx.search(q, 20)
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(It, Ip)
    np.testing.assert_array_equal(Dt, Dp)


def test_inner_product_above_2048_lists():
    rng = np.random.default_rng(44)
    x = rng.standard_normal((60_000, 32)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    q = x[rng.integers(0, 60_000, 500)] + 0.05 * rng.standard_normal((500, 32)).astype(np.float32)
    idx = hb.Index(32, 3000, 40, 0)
    idx.train(x)
    idx.add(x)
    plain = idx.probes(q)
    np.testing.assert_array_equal(_probes(idx, q, "tensor"), plain)
