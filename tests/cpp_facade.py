"""Builds tests/cpp/facade_demo.cpp against include/harmony/Index.h and
libhy.so (shared by the CPU compile test and the GPU run test)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp")
LIBDIR = os.path.join(ROOT, "harmonyclient_b200")


def build(out_dir):
    exe = os.path.join(str(out_dir), "facade_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", LIBDIR,
                    "-lhy", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe
