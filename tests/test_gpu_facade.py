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
