"""The selection rule the tightening and coarse-refine kernels use for their
thresholds (warp_select_bound / kth_bound_stream), restated in numpy and
checked on the CPU: from the minimum and maximum of the ordered 32-bit
values, two 8-bit radix passes below the bits they share; U is the upper edge
of the final bin that holds the k-th value.  U must have at least k values at
or below it (so it bounds the k-th value from above) and lie within
2^(top - 15) of the k-th value in the ordered-bits order."""
import numpy as np
import pytest


def f2o(f):
    """Order-preserving map of float32 to uint32 (the kernels' f2o)."""
    u = np.asarray(f, np.float32).view(np.uint32).astype(np.uint64)
    neg = (u >> 31) == 1
    return np.where(neg, (~u) & 0xFFFFFFFF, u | 0x80000000).astype(np.uint64)


def o2f(o):
    """Inverse of f2o (the kernels' o2f)."""
    o = int(o)
    u = (o & 0x7FFFFFFF) if (o & 0x80000000) else (~o & 0xFFFFFFFF)
    return float(np.array([u], np.uint32).view(np.float32)[0])


def select_bound(v, k):
    v = np.asarray(v, np.uint64)
    mn, mx = int(v.min()), int(v.max())
    if mn == mx:
        return mn, -1
    top = (mn ^ mx).bit_length() - 1
    mask = ~((2 << top) - 1) & 0xFFFFFFFF
    prefix = mn & mask
    rem = k
    for _ in range(2):
        if top < 0:
            break
        shift = top - 7 if top > 7 else 0
        wmask = ((2 << top) - 1) & ~((1 << shift) - 1)
        sel = v[(v & mask) == prefix]
        digits = ((sel & wmask) >> shift).astype(np.int64)
        hist = np.bincount(digits, minlength=256)
        cum = np.cumsum(hist)
        digit = int(np.searchsorted(cum, rem))
        before = int(cum[digit - 1]) if digit > 0 else 0
        prefix |= digit << shift
        mask |= wmask
        rem -= before
        top = shift - 1
    ub = prefix | ((2 << top) - 1) if top >= 0 else prefix
    return ub, top


@pytest.mark.parametrize("seed", range(40))
def test_bound_properties(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 3000))
    k = int(rng.integers(1, n + 1))
    kind = seed % 4
    if kind == 0:
        f = rng.uniform(1e4, 4e5, n)           # L2 distances
    elif kind == 1:
        f = -rng.uniform(0, 1, n)               # inner-product scores (negative)
    elif kind == 2:
        f = rng.integers(0, 50, n).astype(float)  # many ties
    else:
        f = rng.normal(0, 1, n)                 # both signs
    v = f2o(f.astype(np.float32))
    ub, top = select_bound(v, k)
    kth = int(np.sort(v)[k - 1])
    assert int(np.sum(v <= ub)) >= k
    assert ub >= kth
    U = o2f(ub)
    assert not np.isnan(U) and U >= float(np.sort(f.astype(np.float32))[k - 1])
    if top >= 0:
        assert ub - kth < (2 << top)


def test_all_equal_values():
    v = f2o(np.full(100, 3.5, np.float32))
    ub, _ = select_bound(v, 10)
    assert ub == int(v[0])
