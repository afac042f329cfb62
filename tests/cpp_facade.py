"""Builds the C++ programs under tests/cpp/ against include/harmony/Index.h
and libhy.so (shared by the CPU compile tests and the GPU run tests)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "harmonyclient_b200")


def build(out_dir, name="facade_demo"):
    src = os.path.join(ROOT, "tests", "cpp", f"{name}.cpp")
    exe = os.path.join(str(out_dir), name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src, "-o",
                    exe, "-L", LIBDIR, "-lhy", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe
