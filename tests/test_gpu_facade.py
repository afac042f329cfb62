"""The C++ facade (include/harmony/Index.h) driven like the reference's own
callers, checked against the oracle restatement on the same centroids."""
import subprocess

import numpy as np
import pytest

from harmonyclient_b200 import datasets
from oracle import port
from tests.cpp_facade import build
from tests.topk_check import assert_topk_equal, probe_tied_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["plain", "bf16"])
def test_facade_search_matches_oracle(tmp_path, form):
    exe = build(tmp_path)
    x, q = datasets.gmm_float(10_000, 100, seed=11)
    x.tofile(tmp_path / "base.f32")
    q.tofile(tmp_path / "q.f32")
    args = [exe, "128", "100", "10", "10", str(tmp_path / "base.f32"), "10000", str(tmp_path / "q.f32"), "100",
            str(tmp_path / "out")]
    if form == "bf16":
        args.append("bf16")
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    D = np.fromfile(tmp_path / "out.D", np.float32).reshape(100, 10)
    I = np.fromfile(tmp_path / "out.I", np.int64).reshape(100, 10)
    cent = np.fromfile(tmp_path / "out.C", np.float32).reshape(100, 128)
    L = port.build_lists(x, cent)
    P, _ = port.probes(q, cent, 10)
    Do, Io = port.scan_probes(q, L, P, 10)
    assert_topk_equal(Do, Io, D, I, rtol=1e-5, skip_rows=probe_tied_rows(q, cent, P))


def test_reference_style_caller(tmp_path):
    """tests/cpp/benchmark_caller.cpp drives the facade the way the
    reference's drivers drive harmony::Index: the built, file-loaded and
    broadcast-centroid indexes answer alike, nprobe = nlist is exhaustive,
    lists[0] holds the oracle's list 0, the CSV log has the reference's
    columns, and the timing fields are filled."""
    exe = build(tmp_path, "benchmark_caller")
    x, q = datasets.gmm_float(10_000, 100, seed=12)
    x.tofile(tmp_path / "base.f32")
    q.tofile(tmp_path / "q.f32")
    nlist, k = 100, 10
    r = subprocess.run([exe, "128", str(nlist), str(k), str(tmp_path / "base.f32"), "10000", str(tmp_path / "q.f32"),
                        "100", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    for np_ in (1, 4, nlist):
        got = [(np.fromfile(tmp_path / f"D_{np_}_{t}.f32", np.float32).reshape(100, k),
                np.fromfile(tmp_path / f"I_{np_}_{t}.i64", np.int64).reshape(100, k)) for t in "abc"]
        for D, I in got[1:]:
            np.testing.assert_array_equal(I, got[0][1])
            np.testing.assert_array_equal(D, got[0][0])
    D, I = got[0]
    d2 = ((q.astype(np.float64)[:, None, :] - x.astype(np.float64)[None]) ** 2).sum(-1)
    It = np.argsort(d2, axis=1, kind="stable")[:, :k]
    Dt = np.take_along_axis(d2, It, 1).astype(np.float32)
    assert_topk_equal(Dt, It, D, I, rtol=1e-5)
    cent = np.fromfile(tmp_path / "C.f32", np.float32).reshape(nlist, 128)
    L = port.build_lists(x, cent)
    assert sorted(np.fromfile(tmp_path / "list0.i64", np.int64).tolist()) == sorted(
        L.ids[L.offsets[0]:L.offsets[1]].tolist())
    lines = (tmp_path / "log.csv").read_text().strip().split("\n")
    assert len(lines) == 4 and len(lines[0].split(",")) == 28
    assert lines[1].split(",")[1] == "Group   "
    times = [float(t) for t in (tmp_path / "times.txt").read_text().split()]
    assert times[0] > 0 and times[1] > 0 and times[2] >= 0
