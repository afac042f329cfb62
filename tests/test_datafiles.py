"""Dataset, result-file and recall utilities (harmonyclient_b200/datafiles.py)
against the reference's own readers and metrics: the fixtures in
tests/golden/io/ were produced by the reference's src/utils.h code
(tests/golden/make_io_golden.py)."""
import os

import numpy as np
import pytest

from harmonyclient_b200 import datafiles as io

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "io")


@pytest.fixture(scope="module")
def exp():
    return np.load(os.path.join(G, "expected.npz"))


@pytest.mark.parametrize("name", ["a.fvecs", "b.bvecs", "c.txt"])
def test_vector_files_read_as_the_reference_reads_them(exp, name):
    p = os.path.join(G, name)
    assert tuple(io.load_xvecs_info(p)) == tuple(exp[f"{name}_info"])
    np.testing.assert_array_equal(io.load_xvecs(p), exp[f"{name}_all"])
    if not name.endswith(".txt"):
        np.testing.assert_array_equal(io.load_xvecs(p, (2, 4)), exp[f"{name}_2_4"])


def test_row_bounds_are_checked():
    with pytest.raises(ValueError):
        io.load_xvecs(os.path.join(G, "a.fvecs"), (0, 2))
    with pytest.raises(ValueError):
        io.load_xvecs(os.path.join(G, "a.fvecs"), (3, 99))
    with pytest.raises(ValueError):
        io.load_xvecs(os.path.join(G, "x.unknown"))


def test_bvecs_record_layout(tmp_path):
    x = np.arange(40, dtype=np.uint8).reshape(5, 8)
    p = str(tmp_path / "plain.bvecs")
    io.write_bvecs(p, x, bvecs_records=True)
    np.testing.assert_array_equal(io.load_bvecs(p, bvecs_records=True), x)
    q = str(tmp_path / "ref.bvecs")
    io.write_bvecs(q, x)
    np.testing.assert_array_equal(io.load_bvecs(q), x)


@pytest.mark.parametrize("ext", ["bin", "txt"])
def test_result_files_match_the_reference_byte_for_byte(exp, ext, tmp_path):
    p = str(tmp_path / f"r.{ext}")
    io.write_results(exp["res_labels"], exp["res_dist"], p)
    assert open(p, "rb").read() == open(os.path.join(G, f"r.{ext}"), "rb").read()
    lab, dist = io.load_results(os.path.join(G, f"r.{ext}"), 3, 4)
    np.testing.assert_array_equal(lab, exp[f"r_{ext}_labels"])
    np.testing.assert_array_equal(dist, exp[f"r_{ext}_dist"])


@pytest.mark.parametrize("c", range(8))
def test_recall_metrics_equal_the_reference(exp, c):
    nq, k, metric, gt_k = (int(v) for v in exp[f"case{c}_in"])
    args = (exp[f"case{c}_I"], exp[f"case{c}_D"], exp[f"case{c}_GT"], exp[f"case{c}_GD"], nq, k, metric, gt_k)
    got = [io.calculate_recall(*args), io.calculate_recall_loose(*args), io.calculate_r2(*args)]
    np.testing.assert_allclose(np.array(got, np.float32), exp[f"case{c}_out"], rtol=0, atol=0)


def test_k_above_gt_k_rejected():
    I = np.zeros((1, 3), np.int64)
    D = np.ones((1, 3), np.float32)
    with pytest.raises(ValueError):
        io.calculate_recall(I, D, I[:, :2], D[:, :2], 1, 3, io.METRIC_L2, 2)


def test_csv_rows(tmp_path):
    p = str(tmp_path / "stats.csv")
    row = ["sift", 1, 1000, 10, 128, 100, 10, 10, True, False, True, 4, 1, 8, 1, 1, np.float64(1.5), 2.25,
           3.0, np.float32(0.95), np.float32(0.01), 0.0, 1.0, 2.0, 3.0, 1.1, 1.2, 1.3]
    io.append_csv_row(p, row)
    io.append_csv_row(p, row)
    lines = open(p).read().splitlines()
    assert lines[0] == ",".join(io.STATS_COLUMNS)
    assert len(lines) == 3 and lines[1] == lines[2]
    f = lines[1].split(",")
    assert f[8:11] == ["1", "0", "1"]
    assert f[16] == "1.5000000000000000" and f[19] == "0.9500000"


def test_bench_reads_vector_files(tmp_path):
    """bench.py --base-file / --query-file: the first nb / nq rows."""
    import bench

    x = np.arange(60, dtype=np.float32).reshape(10, 6)
    q = np.arange(18, dtype=np.float32).reshape(3, 6)
    io.write_fvecs(str(tmp_path / "b.fvecs"), x)
    io.write_bvecs(str(tmp_path / "q.bvecs"), q.astype(np.uint8))
    xb, qb = bench.file_workload(str(tmp_path / "b.fvecs"), str(tmp_path / "q.bvecs"), 7, 0)
    np.testing.assert_array_equal(xb, x[:7])
    np.testing.assert_array_equal(qb, q)


def test_bench_reads_plain_record_bvecs(tmp_path):
    """A .bvecs file without the reference loader's extra header (the public
    BIGANN layout) is told apart by its size and read whole and in bounds."""
    import bench

    x = np.arange(60, dtype=np.float32).reshape(10, 6)
    q = (np.arange(18, dtype=np.float32).reshape(3, 6) * 7) % 251
    io.write_fvecs(str(tmp_path / "b.fvecs"), x)
    qp = str(tmp_path / "q.bvecs")
    io.write_bvecs(qp, q.astype(np.uint8), bvecs_records=True)
    assert io.bvecs_is_records(qp)
    assert bench._file_info(qp) == (3, 6)
    xb, qb = bench.file_workload(str(tmp_path / "b.fvecs"), qp, 0, 2)
    np.testing.assert_array_equal(qb, q[:2])
    np.testing.assert_array_equal(xb, x)
    rp = str(tmp_path / "r.bvecs")
    io.write_bvecs(rp, q.astype(np.uint8))
    assert not io.bvecs_is_records(rp)
    assert bench._file_info(rp) == (3, 6)


def test_bvecs_bounded_read_matches_whole_read(tmp_path):
    x = (np.arange(7 * 12) % 256).astype(np.uint8).reshape(7, 12)
    for records in (False, True):
        p = str(tmp_path / f"x{int(records)}.bvecs")
        io.write_bvecs(p, x, bvecs_records=records)
        np.testing.assert_array_equal(io.load_bvecs(p, (3, 7), records), x[2:7])
        np.testing.assert_array_equal(io.load_bvecs(p, (1, 1), records), x[:1])
