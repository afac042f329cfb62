"""The arithmetic behind the bf16 form's exactness certificate, checked on the
CPU with numpy float32 (no GPU): integers of magnitude <= 256 are exact in
bf16, and for integer vectors with |x|^2 + |q|^2 < 2^23 the tensor-core form
(|x|^2 + |q|^2) - 2 x.q, accumulated in f32 in any order, equals the plain
scan's sequential f32 sum of (x_j - q_j)^2 bit for bit."""
import numpy as np

from oracle import mlp


def test_integers_up_to_256_are_exact_in_bf16():
    v = np.arange(-256, 257, dtype=np.float32)
    np.testing.assert_array_equal(mlp.bf16_round(v), v.astype(np.float64))
    assert mlp.bf16_round(np.array([257.0], np.float32))[0] != 257.0


def _seq_f32(terms):
    acc = np.float32(0.0)
    for t in terms:
        acc = np.float32(acc + np.float32(t))
    return acc


def test_tensor_form_equals_sequential_sum_in_any_order():
    rng = np.random.default_rng(0)
    for trial in range(300):
        d = int(rng.integers(1, 300))
        lo, hi = (-128, 128) if trial % 2 else (0, 256)
        x = rng.integers(lo, hi + 1, d).astype(np.float32)
        q = rng.integers(lo, hi + 1, d).astype(np.float32)
        xn = _seq_f32(x * x)
        qn = _seq_f32(q * q)
        if float(xn) + float(qn) >= 2 ** 23:
            continue
        plain = _seq_f32((x - q) * (x - q))
        for _ in range(3):
            order = rng.permutation(d)
            ip = _seq_f32((x * q)[order])
            tc = np.float32(np.float32(xn + qn) + np.float32(np.float32(-2.0) * ip))
            assert tc == plain, (trial, d, tc, plain)


def test_certificate_bound_is_needed():
    """Past 2^24 a partial sum can round: the condition is not vacuous."""
    x = np.full(300, 256.0, np.float32)
    xn = _seq_f32(x * x)
    assert float(xn) >= 2 ** 23
    exact = 300 * 256.0 ** 2
    assert float(_seq_f32(np.concatenate([[1.0], x * x]))) != exact + 1.0
