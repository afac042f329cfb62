"""Builds libhy.so (the CUDA engine behind include/hy.h) in-tree for sm_100a,
and harmony_serve (the TCP query server over it).

    python -m harmonyclient_b200.build          # build if sources changed
    python -m harmonyclient_b200.build --force  # rebuild

The library links the CUDA runtime statically so the built file runs on any
host with the NVIDIA driver, and exports only the hy_* C-ABI symbols.
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhy.so")
SERVER = os.path.join(HERE, "harmony_serve")
SOURCES = ["hy_kernels.cu", "hy_batched.cu", "hy_capi.cu", "hy_selftest.cu", "hy_noalloc.cu", "hy_mlp.cu", "hy_lists.cu"]
HEADERS = ["hy_device.cuh", "hy_kernels.cuh", "hy_tc.cuh", "hy_common.cuh", "hy_batched.cuh", "hy_mlp.cuh", "hy_lists.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + ["hy_serve.cpp"]] + [
        os.path.join(ROOT, "include", "hy.h")]
    return files


def stale():
    if not os.path.exists(LIB) or not os.path.exists(SERVER):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(SERVER))
    return any(os.path.getmtime(f) > t for f in _inputs())


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    objs = []
    common = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-I", os.path.join(ROOT, "include")]
    if verbose:
        common += ["-Xptxas", "-v"]
    outdir = os.path.join(HERE, "_build")
    os.makedirs(outdir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(outdir, src.replace(".cu", ".o"))
        subprocess.run(common + ["-c", os.path.join(CSRC, src), "-o", obj], check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp] + objs, check=True)
    os.replace(tmp, LIB)
    build_server()
    return LIB


def build_server():
    """harmony_serve: the TCP query server (csrc/hy_serve.cpp), a host
    program over libhy.so found next to it."""
    tmp = SERVER + ".tmp"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(CSRC, "hy_serve.cpp"), "-o", tmp, "-L", HERE, "-lhy", "-Wl,-rpath,$ORIGIN"],
                   check=True)
    os.replace(tmp, SERVER)
    return SERVER


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
