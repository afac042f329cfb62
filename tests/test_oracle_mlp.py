"""Pins the probe-network oracle on the CPU: its analytic gradient against
central finite differences (float64, no bf16 rounding), its bf16 rounding
against torch's, and its features/labels on hand-made cases."""
import numpy as np
import torch

from oracle import mlp


def _params(rng, scale=0.2):
    p = rng.uniform(-scale, scale, mlp.NPARAM)
    return p


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = _params(rng)
    X = rng.standard_normal((16, mlp.IN))
    t = rng.standard_normal(16)
    _, g = mlp.loss_grad(p, X, t, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(a, b), 6, replace=False)
                          for a, b in [(mlp.W1, mlp.B1), (mlp.B1, mlp.W2), (mlp.W2, mlp.B2), (mlp.B2, mlp.W3),
                                       (mlp.W3, mlp.B3)]] + [np.array([mlp.B3])])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_grad(pp, X, t, rounding=False)[0] - mlp.loss_grad(pm, X, t, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(4)
    a = (rng.standard_normal(100000) * 10.0 ** rng.uniform(-8, 8, 100000)).astype(np.float32)
    a[:4] = [0.0, -0.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8]  # exact ties round to even
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(mlp.bf16_round(a), ref)


def test_features_and_labels():
    s = np.array([[4.0, 4.0, 8.0, 12.0]], np.float32)
    X = mlp.features(s)
    assert np.isclose(X[0, 0], np.log(4.0 + 1e-6))
    assert X[0, 1] == 0.0
    assert np.isclose(X[0, 2], np.log1p(4.0 / (4.0 + 1e-6)))
    assert np.isclose(X[0, 63], np.log1p(8.0 / (4.0 + 1e-6)))  # clamped to the last probe
    probes = np.array([[7, 3, 5, 1], [2, 9, 4, 0]])
    rows = np.array([[3, 7, -1], [2, 2, 2]])
    np.testing.assert_array_equal(mlp.stop_labels(rows, probes), [2, 1])
    np.testing.assert_array_equal(mlp.nprobe_from_prediction([0.0, 1.2, 9.0], 0.5, 64), [2, 4, 64])
