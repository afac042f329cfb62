"""The plain form's list-major scan against its query-major scan.

Both compute every distance with the same arithmetic (block sums from zero in
dimension order, blocks added in order) and keep the k smallest (score, arena
row) keys, so their answers must be equal bit for bit: on the golden cases,
with wide dimension blocks (the multi-chunk kernel), inner product, k from 1
to 256, warm-up thresholds, per-query nprobe, candidate-buffer overflow (the
query-major fallback) and the device-pointer API in graph mode."""
import os

import numpy as np
import pytest
import torch

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets
from tests.golden import cases

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden_index(name):
    c = cases.CASES[name]
    x, q = cases.data(name)
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    idx.centroid_codes = np.load(os.path.join(GOLD, f"{name}.npz"))["centroids"]
    idx.add(x)
    return idx, q, c


def _both(idx, q, k, nprobes=None):
    out = []
    for mode in ("query", "list"):
        idx.set_plain_scan(mode)
        try:
            if nprobes is None:
                D, I = idx.search(q, k)
            else:
                D, I = idx.search_nprobes(q, k, nprobes)
            st = idx.last_stats()
        finally:
            idx.set_plain_scan("auto")
        assert st["list_major"] == (1 if mode == "list" else 0)
        out.append((D, I, st))
    return out


def _equal(a, b):
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[0], b[0])


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small", "exhaustive", "odd_dim"])
def test_list_major_equals_query_major_on_golden_cases(name):
    idx, q, c = _golden_index(name)
    qm, lm = _both(idx, q, c["k"])
    _equal(qm, lm)
    st = lm[2]
    assert st["seg_sums"] > 0 and st["tile_blocks"] > 0


@pytest.mark.parametrize("d,metric", [(200, 1), (420, 1), (200, 0)])
def test_wide_blocks(d, metric):
    """d 200 / 420 with 4 blocks: 64- and 128-float block pitches."""
    x, q = datasets.gmm_dense(30_000, 300, d=d, ncomp=200, seed=d)
    if metric == 0:
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    idx = hb.Index(d, 64, 8, metric)
    idx.train(x)
    idx.add(x)
    qm, lm = _both(idx, q, 20)
    _equal(qm, lm)


@pytest.mark.parametrize("k", [1, 33, 100, 256])
def test_k_range_with_warmup(k):
    x, q = datasets.gmm_uint8(50_000, 500, ncomp=256, seed=11)
    idx = hb.Index(128, 128, 12)
    idx.train(x)
    idx.add(x)
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=k)
    qm, lm = _both(idx, q, k)
    _equal(qm, lm)
    # the warm-up and first-pass thresholds prune: fewer block sums than
    # (query, tile, block) triples
    st = lm[2]
    assert 0 < st["seg_sums"] < st["seg_sums_max"]


def test_per_query_nprobe():
    x, q = datasets.gmm_uint8(40_000, 800, d=64, ncomp=512, sigma=30.0, seed=21)
    idx = hb.Index(64, 64, 32)
    idx.train(x)
    idx.add(x)
    npq = np.random.default_rng(3).integers(1, 33, q.shape[0]).astype(np.int32)
    qm, lm = _both(idx, q, 20, npq)
    _equal(qm, lm)


def test_overflow_is_answered_by_the_query_major_scan():
    """capq 128 < the first pass's candidates of most queries (no warm-up
    threshold: every row of the nearest list is a candidate)."""
    x, q = datasets.gmm_uint8(40_000, 600, d=64, ncomp=64, sigma=30.0, seed=22)
    idx = hb.Index(64, 64, 16)
    idx.train(x)
    idx.add(x)
    idx.set_batch_params(capq=128)
    try:
        qm, lm = _both(idx, q, 50)
    finally:
        idx.set_batch_params(capq=8192)
    _equal(qm, lm)
    assert lm[2]["fallback_queries"] > 0


def test_device_api_in_graph_mode():
    x, q = datasets.gmm_uint8(60_000, 1_000, ncomp=512, seed=23)
    idx = hb.Index(128, 256, 16)
    idx.train(x)
    idx.add(x)
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=50)
    idx.set_plain_scan("query")
    Dq, Iq = idx.search(q, 50)
    idx.set_plain_scan("list")
    idx.set_graph(True)
    try:
        dq = torch.from_numpy(q).cuda()
        dD = torch.empty((q.shape[0], 50), dtype=torch.float32, device="cuda")
        dI = torch.empty((q.shape[0], 50), dtype=torch.int64, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        for _ in range(3):  # runs, captures, replays
            dD.fill_(-1.0)
            idx.search_device(q.shape[0], dq.data_ptr(), 50, dD.data_ptr(), dI.data_ptr(), s)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(dI.cpu().numpy(), Iq)
            np.testing.assert_array_equal(dD.cpu().numpy(), Dq)
        st = idx.last_stats()
        assert st["list_major"] == 1 and st["kernel_launches"] == 2
    finally:
        idx.set_graph(False)
        idx.set_plain_scan("auto")


def test_ip_triangle_window_matches_reference():
    """OPT_TRIANGLE on clustered unit-norm data (tests/golden/ip_tri.npz, the
    reference's own answer at that opt level): the list-major scan skips the
    rows outside each (query, list) window and returns the reference's
    answer, which is also the exact (OPT_NONE) one."""
    from tests.topk_check import assert_topk_equal, probe_tied_rows
    idx, q, c = _golden_index("ip_tri")
    g = np.load(os.path.join(GOLD, "ip_tri.npz"))
    idx.set_plain_scan("list")
    try:
        D0, I0 = idx.search(q, c["k"])
        st0 = idx.last_stats()
        idx.opt_level = hb.OPT_TRIANGLE
        D1, I1 = idx.search(q, c["k"])
        st1 = idx.last_stats()
    finally:
        idx.opt_level = hb.OPT_NONE
        idx.set_plain_scan("auto")
    tied = probe_tied_rows(q, g["centroids"], g["probes"], 0)
    assert_topk_equal(g["D"], g["I"], D1, I1, rtol=1e-5, metric=0, skip_rows=tied)
    assert_topk_equal(D0, I0, D1, I1, rtol=1e-5, metric=0)
    # the window skipped most of the probed rows' work
    assert st1["seg_sums"] < 0.5 * st0["seg_sums"], (st1["seg_sums"], st0["seg_sums"])
    assert st1["tile_blocks"] < st0["tile_blocks"]


def test_l2_triangle_window_changes_no_answer():
    """L2 with OPT_TRIANGLE: the list-major scan skips rows whose distance to
    their centroid is too far from the query's (an exact prune); the answer
    is the same bit for bit, and on tight clusters work is skipped."""
    c = cases.CASES["ip_tri"]
    x, q = cases.data("ip_tri")  # tight clusters, one per list
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], hb.METRIC_L2)
    idx.train(x)
    idx.add(x)
    idx.set_plain_scan("list")
    try:
        D0, I0 = idx.search(q, c["k"])
        st0 = idx.last_stats()
        idx.opt_level = hb.OPT_TRIANGLE
        D1, I1 = idx.search(q, c["k"])
        st1 = idx.last_stats()
    finally:
        idx.opt_level = hb.OPT_NONE
        idx.set_plain_scan("auto")
    np.testing.assert_array_equal(I1, I0)
    np.testing.assert_array_equal(D1, D0)
    assert st1["tile_blocks"] < st0["tile_blocks"]


@pytest.mark.parametrize("case", ["empty_lists", "one_query", "one_list", "k_beyond_rows", "odd_batch"])
def test_edge_cases_equal_query_major(case):
    rng = np.random.default_rng(41)
    if case == "empty_lists":
        # centroids far from every row leave most lists empty
        x = rng.integers(0, 50, (3_000, 32)).astype(np.float32)
        cent = np.vstack([x[:5], np.full((59, 32), 1e4, np.float32) + rng.random((59, 32)).astype(np.float32)])
        idx = hb.Index(32, 64, 16)
        idx.centroid_codes = cent
        idx.add(x)
        q, k = x[::7][:300], 10
    elif case == "one_query":
        x, q = datasets.gmm_uint8(20_000, 1, d=64, ncomp=64, seed=42)
        idx = hb.Index(64, 32, 32)
        idx.train(x)
        idx.add(x)
        k = 20
    elif case == "one_list":
        x, q = datasets.gmm_uint8(5_000, 200, d=48, ncomp=8, seed=43)
        idx = hb.Index(48, 1, 1)
        idx.train(x)
        idx.add(x)
        k = 50
    elif case == "k_beyond_rows":
        x, q = datasets.gmm_uint8(2_000, 100, d=16, ncomp=16, seed=44)
        idx = hb.Index(16, 64, 2)
        idx.train(x)
        idx.add(x)
        k = 256
    else:
        x, q = datasets.gmm_uint8(30_000, 333, d=96, ncomp=128, seed=45)
        idx = hb.Index(96, 48, 12)
        idx.train(x)
        idx.add(x)
        idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=7)
        k = 7
    qm, lm = _both(idx, q, k)
    _equal(qm, lm)
    if case == "k_beyond_rows":
        assert (lm[1][:, -1] == -1).all()
