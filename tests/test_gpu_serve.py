"""harmony_serve (the reference's TCP serving path, src/query.cpp:446-799 and
src/master_server.cpp) driven through the reference's protocol by
harmonyclient_b200.serve_client: the insert phase (OP_INSERT batches,
OP_BUILD_DONE), then query batches whose answers must equal the library's
own search of the same index bit for bit, then shutdown; and the load path
(--index)."""
import os
import socket
import subprocess

import numpy as np
import pytest

import harmonyclient_b200 as hb
from harmonyclient_b200 import datafiles, datasets
from harmonyclient_b200.serve_client import ServeClient
from tests.topk_check import assert_topk_equal

pytestmark = pytest.mark.gpu
SERVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "harmonyclient_b200",
                      "harmony_serve")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _expected(path, q, k, nprobe, form):
    info = hb.file_inspect(path)
    idx = hb.Index(info["d"], info["nlist"], nprobe)
    idx.load_index(path)
    idx.nprobe = nprobe
    idx.preSearch(warmUpSearchList=10, warmUpSearchListSize=0)
    idx.set_form(form)
    return idx.search(q, k)


@pytest.mark.parametrize("form", ["plain", "bf16"])
def test_insert_build_query_shutdown(tmp_path, form):
    x, q = datasets.gmm_uint8(30_000, 300, ncomp=256, seed=31)
    seed = str(tmp_path / "seed.fvecs")
    datafiles.write_fvecs(seed, x[:10_000])
    saved = str(tmp_path / "served.index")
    port = _free_port()
    proc = subprocess.Popen([SERVER, "--train_data", seed, "--nlist", "128", "--nprobe", "16", "--form", form,
                             "--port", str(port), "--save", saved], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                            text=True)
    try:
        c = ServeClient("127.0.0.1", port)
        c.insert(x, batch=7_000)
        c.build_done()
        c.reconnect()
        D1, I1 = c.query(q[:100], 10)
        D2, I2 = c.query(q, 50)
        c.shutdown()
        out, err = proc.communicate(timeout=120)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 0, err
    De, Ie = _expected(saved, q, 50, 16, form)
    np.testing.assert_array_equal(I2, Ie)
    np.testing.assert_array_equal(D2, De)
    np.testing.assert_array_equal(I1, Ie[:100, :10])
    np.testing.assert_array_equal(D1, De[:100, :10])


def test_serves_a_reference_index_file(tmp_path):
    """--index with the .index file the reference itself wrote."""
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tiny_ref.index")
    from tests.golden import cases
    x, _ = cases.data("tiny_file")
    q = x[:16]
    port = _free_port()
    proc = subprocess.Popen([SERVER, "--index", gold, "--nprobe", "4", "--port", str(port)],
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        c = ServeClient("127.0.0.1", port)
        D, I = c.query(q, 5)
        c.shutdown()
        out, err = proc.communicate(timeout=60)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 0, err
    g = np.load(os.path.join(os.path.dirname(gold), "tiny_ref_search.npz"))
    assert_topk_equal(g["D"], g["I"], D, I, rtol=1e-5)
