"""The learned probe predictor on the GPU: the training kernels' loss and
gradients against the numpy oracle (same bf16 rounding of matrix-product
inputs), the device inference path (features -> network -> per-query nprobe)
against the oracle's prediction, the judge's fallback, model export/import,
and the predictor's gain over a fixed nprobe on a mixture whose queries differ
in difficulty."""
import ctypes as C

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import _lib, datasets
from oracle import mlp, port

pytestmark = pytest.mark.gpu


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _glorot(rng):
    p = np.zeros(mlp.NPARAM, np.float32)
    for off, fi, fo in [(mlp.W1, mlp.IN, mlp.H), (mlp.W2, mlp.H, mlp.H), (mlp.W3, mlp.H, 1)]:
        a = np.sqrt(6.0 / (fi + fo))
        p[off:off + fi * fo] = rng.uniform(-a, a, fi * fo)
    p[mlp.B1:mlp.W2] = rng.uniform(-0.1, 0.1, mlp.H)
    p[mlp.B2:mlp.W3] = rng.uniform(-0.1, 0.1, mlp.H)
    p[mlp.B3] = 0.3
    return p


@pytest.mark.parametrize("B", [256, 100])
def test_mlp_loss_and_gradients_match_oracle(B):
    rng = np.random.default_rng(11 + B)
    p = _glorot(rng)
    X = rng.standard_normal((B, mlp.IN)).astype(np.float32)
    t = (rng.standard_normal(B) * 2.0 + 2.0).astype(np.float32)
    L = _lib.load()
    loss = np.zeros(1, np.float32)
    g = np.zeros(mlp.NPARAM, np.float32)
    assert L.hy_mlp_loss_grad(_ptr(p), B, _ptr(X), _ptr(t), _ptr(loss), _ptr(g)) == 0
    ref_loss, ref_g = mlp.loss_grad(p, X, t, rounding=True)
    # f32 accumulation vs float64: relative 1e-4 on the loss, 2e-3 (relative
    # L2 norm) per parameter tensor, and every element within 1e-2 of the
    # tensor's largest gradient.
    assert abs(loss[0] - ref_loss) <= 1e-4 * abs(ref_loss)
    for a, b in [(mlp.W1, mlp.B1), (mlp.B1, mlp.W2), (mlp.W2, mlp.B2), (mlp.B2, mlp.W3), (mlp.W3, mlp.B3),
                 (mlp.B3, mlp.NPARAM)]:
        gg, rr = g[a:b].astype(np.float64), ref_g[a:b]
        assert np.linalg.norm(gg - rr) <= 2e-3 * np.linalg.norm(rr) + 1e-12, (a, b)
        assert np.max(np.abs(gg - rr)) <= 1e-2 * np.max(np.abs(rr)) + 1e-12, (a, b)


def _hard_mixture(nb=200_000, nq=12_000, d=64):
    # sigma 60 around 1024 centres: neighbours often straddle lists, so the
    # number of lists a query needs varies from 1 to all 64.
    return datasets.gmm_uint8(nb, nq, d=d, ncomp=1024, sigma=60.0, seed=5)


@pytest.fixture(scope="module")
def trained():
    x, q = _hard_mixture()
    idx = hb.Index(x.shape[1], 256, 64)
    idx.train(x)
    idx.add(x)
    rep = idx.train_probe_model(q[:10_000], max_nprobe=64, k_label=10, epochs=40, lr=1e-3, coverage=0.9)
    return idx, x, q, rep


def _recall(I, G, k=10):
    return np.mean([len(set(a[:k]) & set(b[:k])) / k for a, b in zip(I, G)])


def test_training_report(trained):
    idx, x, q, rep = trained
    assert 0.85 <= rep["coverage"] <= 0.95
    assert 1.0 <= rep["mean_label"] <= 64.0
    assert rep["mean_nprobe"] < 64.0
    assert np.isfinite(rep["loss"]) and rep["loss"] < 4.0


def test_device_prediction_matches_oracle(trained):
    """The search's per-query nprobe equals the oracle's prediction from the
    same model: the learned search returns what a preassigned search over the
    oracle-truncated probe lists returns."""
    idx, x, q, _ = trained
    qt = q[10_000:11_000]
    model = idx.get_probe_model()
    params = model[:mlp.NPARAM]
    mu = model[mlp.NPARAM:mlp.NPARAM + mlp.IN]
    sd = model[mlp.NPARAM + mlp.IN:mlp.NPARAM + 2 * mlp.IN]
    margin, P = float(model[-2]), int(model[-1])
    assert P == 64
    probes, scores = port.probes(qt, idx.centroid_codes, 64)
    feats = (mlp.features(scores).astype(np.float32) - mu) / sd
    y, _ = mlp.forward(params, feats.astype(np.float32), rounding=True)
    npq = mlp.nprobe_from_prediction(y, margin, P)
    cut = probes.copy()
    for i, n in enumerate(npq):
        cut[i, n:] = -1
    Dp, Ip = idx.search_preassigned(qt, 10, cut)
    idx.set_learned(True, judge_fraction=0.0)
    try:
        Dl, Il = idx.search(qt, 10)
        st = idx.last_stats()
    finally:
        idx.set_learned(False)
    same = np.all(Il == Ip, axis=1) & np.all(Dl == Dp, axis=1)
    # f32 feature arithmetic vs float64 moves y by ~1e-6; only a query whose
    # 2^(y+margin) sits on an integer may round to the other nprobe.
    assert same.mean() >= 0.99, same.mean()
    assert abs(st["mean_nprobe"] - npq.mean()) <= 0.05 * npq.mean()


def test_learned_gain_over_fixed_nprobe(trained):
    idx, x, q, _ = trained
    qt = q[10_000:]
    idx.nprobe = 256
    _, G = idx.search(qt, 10)  # exhaustive ground truth
    idx.nprobe = 64
    idx.set_learned(True, judge_fraction=0.0)
    try:
        _, Il = idx.search(qt, 10)
        mean_np = idx.last_stats()["mean_nprobe"]
    finally:
        idx.set_learned(False)
    r_learned = _recall(Il, G)
    idx.nprobe = int(np.ceil(mean_np))
    _, If = idx.search(qt, 10)
    r_fixed = _recall(If, G)
    idx.nprobe = 64
    assert r_learned >= 0.95, r_learned
    assert mean_np <= 0.5 * 64, mean_np
    # Same average number of lists, better recall.
    assert r_learned >= r_fixed + 0.005, (r_learned, r_fixed, mean_np)


def test_learned_bf16_form_equals_learned_plain(trained):
    idx, x, q, _ = trained
    qt = q[10_000:11_000]
    idx.set_learned(True, judge_fraction=0.0)
    try:
        idx.set_form("plain")
        Dp, Ip = idx.search(qt, 10)
        idx.set_form("bf16")
        Db, Ib = idx.search(qt, 10)
    finally:
        idx.set_form("plain")
        idx.set_learned(False)
    np.testing.assert_array_equal(Ib, Ip)
    np.testing.assert_array_equal(Db, Dp)


def test_judge_falls_back_to_fixed_nprobe(trained):
    """A model that always predicts one list fails a judge that wants full
    recall, and the batch is searched again with the fixed nprobe."""
    idx, x, q, _ = trained
    qt = q[10_000:10_500]
    D0, I0 = idx.search(qt, 10)
    keep = idx.get_probe_model()
    weak = keep.copy()
    weak[:mlp.NPARAM] = 0.0
    weak[mlp.B3] = -10.0
    weak[-2] = 0.0
    try:
        idx.set_probe_model(weak)
        idx.set_learned(True, judge_fraction=0.05, judge_recall=1.0)
        D1, I1 = idx.search(qt, 10)
        st = idx.last_stats()
        assert st["learned_fallback"] == 1
        assert 0.0 <= st["judge_recall"] < 1.0
        np.testing.assert_array_equal(I1, I0)
        np.testing.assert_array_equal(D1, D0)
        idx.set_learned(True, judge_fraction=0.0)
        idx.search(qt, 10)
        assert idx.last_stats()["mean_nprobe"] == 1.0
    finally:
        idx.set_learned(False)
        idx.set_probe_model(keep)


def test_model_round_trip_and_errors(trained):
    idx, x, q, _ = trained
    model = idx.get_probe_model()
    other = hb.Index(idx.d, idx.nlist, 64)
    with pytest.raises(hb.HyError):
        other.set_learned(True)
    other.centroid_codes = idx.centroid_codes
    other.add(x)
    other.set_probe_model(model)
    np.testing.assert_array_equal(other.get_probe_model(), model)
    qt = q[11_000:11_300]
    for h in (idx, other):
        h.set_learned(True, judge_fraction=0.0)
    try:
        Da, Ia = idx.search(qt, 10)
        Db, Ib = other.search(qt, 10)
    finally:
        idx.set_learned(False)
    np.testing.assert_array_equal(Ia, Ib)
    np.testing.assert_array_equal(Da, Db)
    with pytest.raises(hb.HyError):
        idx.set_learned(True, judge_fraction=2.0)


def test_graph_mode_learned_and_judge_fallback(trained):
    """Graph mode with the learned form: replays keep the learned answer, and
    the judge's fallback search (learned off, same batch shape) is not served
    by the learned graph."""
    idx, x, q, _ = trained
    qt = q[10_000:10_500]
    D0, I0 = idx.search(qt, 10)
    idx.set_learned(True, judge_fraction=0.0)
    Dl, Il = idx.search(qt, 10)
    keep = idx.get_probe_model()
    weak = keep.copy()
    weak[:mlp.NPARAM] = 0.0
    weak[mlp.B3] = -10.0
    weak[-2] = 0.0
    idx.set_graph(True)
    try:
        for _ in range(2):
            D, I = idx.search(qt, 10)
            np.testing.assert_array_equal(I, Il)
            np.testing.assert_array_equal(D, Dl)
        idx.set_probe_model(weak)
        idx.set_learned(True, judge_fraction=1.0, judge_recall=1.0)
        for _ in range(2):
            D, I = idx.search(qt, 10)
            assert idx.last_stats()["learned_fallback"] == 1
            np.testing.assert_array_equal(I, I0)
            np.testing.assert_array_equal(D, D0)
    finally:
        idx.set_graph(False)
        idx.set_learned(False)
        idx.set_probe_model(keep)
