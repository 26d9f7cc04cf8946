"""Compiles tests/cpp/cg_sense_driver.cpp against include/gadgetron_b200.hpp
and libgadgetron_b200.so (test infrastructure)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_driver(out_path: str) -> str:
    libdir = os.path.join(ROOT, "gadgetron_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "cg_sense_driver.cpp"), "-o", out_path,
           "-L", libdir, "-lgadgetron_b200", "-Wl,-rpath," + libdir,
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    subprocess.check_call(cmd)
    return out_path
