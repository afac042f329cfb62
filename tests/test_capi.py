"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/hy.h declares, reads the reference's .index format, and fails with
clear status codes where a GPU would be needed."""
import ctypes as C
import os

import pytest

from harmonyclient_b200 import _lib, file_inspect
from harmonyclient_b200._lib import HyError

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_exports_every_declared_symbol():
    L = _lib.load()
    names = _lib.declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"libhy.so does not export {n}"


def test_version_and_error_string():
    L = _lib.load()
    assert b"sm_100a" in L.hy_version()
    assert isinstance(L.hy_last_error(), bytes)


def test_create_argument_validation():
    L = _lib.load()
    h = C.c_void_p()
    assert L.hy_index_create(0, 10, 1, 1, 0, 4, 0, C.byref(h)) == _lib.HY_ERR_ARG
    assert L.hy_index_create(8, 10, 1, 5, 0, 4, 0, C.byref(h)) == _lib.HY_ERR_ARG
    assert L.hy_index_create(8, 10, 1, 1, 9, 4, 0, C.byref(h)) == _lib.HY_ERR_ARG
    assert L.hy_index_create(8, 10, 1, 1, 0, 99, 0, C.byref(h)) == _lib.HY_ERR_ARG
    assert L.hy_index_create(8, 10, 1, 1, 0, 4, 0, None) == _lib.HY_ERR_ARG


def test_null_handles_rejected():
    L = _lib.load()
    assert L.hy_index_search(None, 1, None, 1, None, None) == _lib.HY_ERR_ARG
    assert L.hy_index_add(None, 1, None) == _lib.HY_ERR_ARG
    assert L.hy_index_destroy(None) == _lib.HY_OK


def test_file_inspect_reads_reference_index():
    info = file_inspect(os.path.join(GOLD, "tiny_ref.index"))
    assert info["d"] == 8 and info["nlist"] == 8 and info["metric"] == 1
    assert info["ntotal"] == 500
    assert 1 <= info["nonempty_lists"] <= 8


def test_file_inspect_rejects_truncated(tmp_path):
    src = open(os.path.join(GOLD, "tiny_ref.index"), "rb").read()
    p = tmp_path / "trunc.index"
    p.write_bytes(src[: len(src) // 2])
    with pytest.raises(HyError) as e:
        file_inspect(p)
    assert e.value.code == _lib.HY_ERR_IO
    with pytest.raises(HyError):
        file_inspect(tmp_path / "missing.index")


@pytest.mark.parametrize("name", ["facade_demo", "benchmark_caller"])
def test_cpp_facade_compiles(tmp_path, name):
    """include/harmony/Index.h compiles as C++17 (warnings as errors) and
    links against libhy.so, for a minimal caller and for one that uses every
    public member the reference's drivers touch."""
    from tests.cpp_facade import build
    exe = build(tmp_path, name)
    assert os.path.exists(exe)


def test_server_builds_and_checks_its_arguments():
    """harmony_serve is built next to libhy.so and refuses a call without
    exactly one of --index / --train_data (no GPU needed)."""
    import subprocess

    from harmonyclient_b200 import build
    exe = build.build_server()
    r = subprocess.run([exe, "--port", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "exactly one of" in r.stderr
    r = subprocess.run([exe, "--index", "a", "--train_data", "b"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
