"""Build recipe for libgadgetron_b200.so (sm_100a only).

Every CUDA source under csrc/ is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked, with cuFFT, into one
shared library placed next to this file (in-tree, so it travels with the
repository).  Run ``python gadgetron_b200/build.py`` (this file does not
import the package, which needs the built library).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgadgetron_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                 "-I" + os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.hpp")) +
                  glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
    cmd = [NVCC] + CFLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), _sources()))
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + [
        "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
        "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas-v" in sys.argv))
