"""Graph mode (the device-pointer search captured once in a CUDA graph and
replayed) and the bf16 form's autotuner: both must leave every answer as the
plain search gives it."""
import numpy as np
import pytest
import torch

import harmonyclient_b200 as hb
from harmonyclient_b200 import datasets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def index():
    x, q = datasets.gmm_uint8(50_000, 600, d=128, ncomp=512, sigma=25.0, seed=31)
    idx = hb.Index(128, 128, 16)
    idx.train(x)
    idx.add(x)
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=50)
    return idx, x, q


@pytest.mark.parametrize("form", ["plain", "bf16"])
@pytest.mark.parametrize("own_stream", [False, True])
def test_graph_replay_equals_direct_search(index, form, own_stream):
    idx, x, q = index
    k = 50
    D0, I0 = idx.search(q, k)
    st = torch.cuda.Stream() if own_stream else torch.cuda.default_stream()
    sp = st.cuda_stream
    dq = torch.from_numpy(q).cuda()
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    idx.set_form(form)
    idx.set_graph(True)
    try:
        replayed = []
        for rep in range(3):
            dD.fill_(0)
            dI.fill_(0)
            torch.cuda.synchronize()
            idx.search_device(q.shape[0], dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(), sp)
            st.synchronize()
            replayed.append(idx.last_stats()["graph_replayed"])
            np.testing.assert_array_equal(dI.cpu().numpy(), I0)
            np.testing.assert_array_equal(dD.cpu().numpy(), D0)
        assert replayed == [0, 1, 1]
        # A parameter change retires the graph; the next call captures anew.
        idx.nprobe = 8
        D8, I8 = idx.search(q, k)
        idx.search_device(q.shape[0], dq.data_ptr(), k, dD.data_ptr(), dI.data_ptr(), sp)
        st.synchronize()
        assert idx.last_stats()["graph_replayed"] == 0
        np.testing.assert_array_equal(dI.cpu().numpy(), I8)
    finally:
        idx.nprobe = 16
        idx.set_graph(False)
        idx.set_form("plain")


def test_graph_with_per_query_nprobe(index):
    idx, x, q = index
    k = 20
    npq = np.random.default_rng(2).integers(1, 17, q.shape[0]).astype(np.int32)
    idx.set_form("bf16")
    D0, I0 = idx.search_nprobes(q, k, npq)
    dq = torch.from_numpy(q).cuda()
    dn = torch.from_numpy(npq).cuda()
    dD = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    dI = torch.empty((q.shape[0], k), dtype=torch.int64, device="cuda")
    idx.set_graph(True)
    try:
        for _ in range(2):
            dI.fill_(0)
            idx.search_nprobes_device(q.shape[0], dq.data_ptr(), k, dn.data_ptr(), 16, dD.data_ptr(), dI.data_ptr(),
                                      0)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(dI.cpu().numpy(), I0)
            np.testing.assert_array_equal(dD.cpu().numpy(), D0)
        assert idx.last_stats()["graph_replayed"] == 1
    finally:
        idx.set_graph(False)
        idx.set_form("plain")


def test_autotune_keeps_answers(index):
    idx, x, q = index
    D0, I0 = idx.search(q, 50)
    idx.set_form("bf16")
    try:
        rep = idx.autotune(q, 50, reps=2)
        assert len(rep) == 6 and all(r[3] for r in rep), rep
        chosen = idx.batch_params()
        best = min(rep, key=lambda r: r[2])
        assert (chosen["row_slice"], chosen["capq"]) == (best[0], best[1])
        D1, I1 = idx.search(q, 50)
    finally:
        idx.set_form("plain")
    np.testing.assert_array_equal(I1, I0)
    np.testing.assert_array_equal(D1, D0)


def test_autotune_needs_bf16_form(index):
    idx, x, q = index
    with pytest.raises(hb.HyError):
        idx.autotune(q[:10], 10)


def test_host_search_replays_the_graph(index):
    """The host-pointer search in graph mode: upload, replayed search,
    download; every answer equals the plain search's."""
    idx, x, q = index
    D0, I0 = idx.search(q, 30)
    idx.set_form("bf16")
    idx.set_graph(True)
    try:
        replayed = []
        for _ in range(3):
            D, I = idx.search(q, 30)
            replayed.append(idx.last_stats()["graph_replayed"])
            np.testing.assert_array_equal(I, I0)
            np.testing.assert_array_equal(D, D0)
        assert replayed == [0, 1, 1]
        idx.nprobe = 8
        D8, I8 = idx.search(q, 30)
        assert idx.last_stats()["graph_replayed"] == 0
    finally:
        idx.nprobe = 16
        idx.set_graph(False)
        idx.set_form("plain")
    idx.nprobe = 8
    try:
        Dp8, Ip8 = idx.search(q, 30)
    finally:
        idx.nprobe = 16
    np.testing.assert_array_equal(I8, Ip8)
    np.testing.assert_array_equal(D8, Dp8)
