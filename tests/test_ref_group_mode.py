"""The reference's GROUP mode with pruning (its default distributed mode,
src/Index.cpp:1053-1187 with src/node.cpp:679-1203), its MPI ranks run as
threads by oracle/ref_mpi_threads.cpp: it completes and returns the answer of
the reference's ORIGINAL search on the same index.  This is the CPU baseline
of the multi-rank path; no GPU is involved."""
import numpy as np
import pytest

from oracle import ref
from tests.golden import cases
from tests.topk_check import assert_topk_equal, probe_tied_rows

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref (the reference library) not built")


@pytest.mark.parametrize("name,workers,group,team,block", [("c1", 4, 2, 2, 4), ("int_small", 2, 2, 1, 4),
                                                           ("c1", 6, 3, 3, 2)])
def test_group_mode_equals_original(name, workers, group, team, block):
    c = cases.CASES[name]
    x, q = cases.data(name)
    g = np.load(f"tests/golden/{name}.npz")
    R = ref.RefIndex(c["d"], c["nlist"], c["nprobe"])
    R.set_centroids(g["centroids"])
    R.add(x)
    nq = q.shape[0] // (group * block) * (group * block)  # the reference needs nq divisible by group x block
    q = q[:nq]
    D, I, secs = R.search_group(q, c["k"], workers=workers, group=group, team=team, block=block,
                                threads_per_rank=2)
    assert secs > 0
    Do, Io = R.search(q, c["k"])
    tied = probe_tied_rows(q, g["centroids"], g["probes"][:nq])
    assert_topk_equal(Do, Io, D, I, rtol=0.0 if name == "int_small" else 1e-5, skip_rows=tied)
