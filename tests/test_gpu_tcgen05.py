"""The tensor-core plumbing on its own: one 128 x 128 x 128 bf16 tile
product through shared-memory descriptors, tcgen05.mma, TMEM and tcgen05.ld,
checked exactly (small integers are exact in bf16 and in the f32
accumulator)."""
import ctypes as C

import numpy as np
import pytest

from harmonyclient_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(A, B):
    L = _lib.load()
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    D = np.zeros((128, 128), np.float32)
    _lib.check(L.hy_selftest_tcgen05(A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p),
                                     D.ctypes.data_as(C.c_void_p)))
    return D


def test_identity_picks_rows():
    rng = np.random.default_rng(0)
    A = rng.integers(-8, 9, (128, 128)).astype(np.float32)
    D = _run(A, np.eye(128, dtype=np.float32))
    np.testing.assert_array_equal(D, A)


def test_integer_product_exact():
    rng = np.random.default_rng(1)
    A = rng.integers(0, 256, (128, 128)).astype(np.float32)
    B = rng.integers(0, 256, (128, 128)).astype(np.float32)
    D = _run(A, B)
    np.testing.assert_array_equal(D, (A.astype(np.int64) @ B.astype(np.int64).T).astype(np.float32))
