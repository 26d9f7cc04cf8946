"""Build recipe for oracle/_ref/libgbref.so: the reference's own GPU
reconstruction path, compiled from its sources where they lie, plus the
C-ABI driver oracle/ref_driver.cu.  Test infrastructure only: the product
never loads the result.

Usage:  python oracle/build_ref.py [--reference DIR] [--jobs N] [--force]

The reference's build system (CMake) is not run.  Its GPU path needs only a
few Boost headers, which oracle/ref_shim/ stands in for with the standard
library, and one CMake-generated header (core_defines.h), which this script
writes from toolboxes/core/core_defines.h.in with the CUDA flag set.  Two
adjustments let the unmodified sources build with this image's toolchain
(nvcc 12.9 / CCCL 2.8 / g++ 13):

* toolboxes/core/gpu/cuNDArray_operators.cu repeats, on its definitions, the
  default template argument (`class = std::enable_if_t<...>`) that
  cuNDArray_operators.h already gives; g++ 13 rejects the redefinition.  A
  copy with those 16 repeated defaults dropped is generated under
  oracle/_ref/gen/ and compiled instead (the header keeps them, so the
  operators resolve exactly as before).
* toolboxes/nfft/gpu/cuGriddingConvolution.cu gets oracle/ref_shim/
  gb_ref_scan.h forced in, which resolves one inclusive_scan call that CCCL
  2.8 makes ambiguous.

Outputs go only to oracle/_ref/ (git-ignored; it travels with the working
tree to a GPU machine, where the library is loaded without rebuilding).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "ref_shim")
LIB = os.path.join(OUT, "libgbref.so")

# The reference's GPU reconstruction path (toolboxes/CMakeLists.txt's
# gadgetron_toolbox_gpu members that cuNFFT, the SENSE operator and the CG
# solver need).
SOURCES = [
    "toolboxes/nfft/gpu/cuNFFT.cu",
    "toolboxes/nfft/gpu/cuGriddingConvolution.cu",
    "toolboxes/fft/gpu/cuNDFFT.cpp",
    "toolboxes/fft/gpu/cuNDFFT.cu",
    "toolboxes/core/gpu/cuNDArray_utils.cu",
    "toolboxes/core/gpu/cuNDArray_elemwise.cu",
    "toolboxes/core/gpu/cuNDArray_operators.cu",
    "toolboxes/core/gpu/cuNDArray_blas.cu",
    "toolboxes/core/gpu/cuNDArray_reductions.cu",
    "toolboxes/core/gpu/cudaDeviceManager.cpp",
    "toolboxes/core/gpu/cuSparseMatrix.cu",
    "toolboxes/mri/pmri/gpu/sense_utilities.cu",
    "toolboxes/mri/pmri/gpu/cuSenseOperator.cu",
    "toolboxes/mri/pmri/gpu/cuNonCartesianSenseOperator.cu",
    "toolboxes/log/log.cpp",
]

INCLUDE_DIRS = [
    "toolboxes/core", "toolboxes/core/gpu", "toolboxes/core/cpu", "toolboxes/core/cpu/math",
    "toolboxes/nfft", "toolboxes/nfft/gpu", "toolboxes/fft/gpu", "toolboxes/fft/cpu",
    "toolboxes/operators", "toolboxes/operators/gpu", "toolboxes/solvers", "toolboxes/solvers/gpu",
    "toolboxes/mri/pmri/gpu", "toolboxes/mri/core", "toolboxes/log", "core",
]

NVCC_FLAGS = [
    "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "--expt-extended-lambda", "-w",
    "-Wno-deprecated-declarations", "-diag-suppress=20012,20014,20015",
]

REPEATED_DEFAULT = re.compile(
    r"class = std::enable_if_t<enable_operator_v<T>>|class = std::enable_if_t<enable_operator<T>\(\)>")


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _generate(ref):
    gen = os.path.join(OUT, "gen")
    os.makedirs(gen, exist_ok=True)
    with open(os.path.join(ref, "toolboxes/core/core_defines.h.in")) as f:
        txt = f.read()
    _write_if_changed(os.path.join(gen, "core_defines.h"), txt.replace("@GADGETRON_CUDA_FOUND_BOOL@", "1"))
    with open(os.path.join(ref, "toolboxes/core/gpu/cuNDArray_operators.cu")) as f:
        src = f.read()
    fixed, n = REPEATED_DEFAULT.subn("class", src)
    if n == 0:
        raise RuntimeError("cuNDArray_operators.cu: expected repeated default template arguments not found")
    _write_if_changed(os.path.join(gen, "cuNDArray_operators.cu"), fixed)
    return gen


def _write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


def _compile(job):
    cmd, obj, log = job
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout)
    return obj, r.returncode, r.stdout


def build(reference="/root/reference", jobs=None, force=False, quiet=False):
    ref = os.path.abspath(reference)
    if not os.path.isdir(os.path.join(ref, "toolboxes/nfft/gpu")):
        raise RuntimeError("reference sources not found under %s" % ref)
    nvcc = _nvcc()
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    gen = _generate(ref)
    incs = ["-I" + SHIM, "-I" + gen] + ["-I" + os.path.join(ref, d) for d in INCLUDE_DIRS]
    base = [nvcc] + NVCC_FLAGS + ["-include", os.path.join(SHIM, "gb_ref_shim.h")] + incs
    work = []
    objs = []
    for rel in SOURCES:
        src = os.path.join(ref, rel)
        extra = []
        if rel.endswith("cuNDArray_operators.cu"):
            src = os.path.join(gen, "cuNDArray_operators.cu")
        if rel.endswith("cuGriddingConvolution.cu"):
            extra = ["-include", os.path.join(SHIM, "gb_ref_scan.h")]
        obj = os.path.join(OUT, "obj", rel.replace("/", "_") + ".o")
        objs.append(obj)
        deps = [src, os.path.abspath(__file__)]
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            work.append((base + extra + ["-x", "cu", "-c", src, "-o", obj], obj, obj + ".log"))
    drv = os.path.join(HERE, "ref_driver.cu")
    drv_obj = os.path.join(OUT, "obj", "ref_driver.o")
    objs.append(drv_obj)
    if force or not os.path.exists(drv_obj) or os.path.getmtime(drv_obj) < max(
            os.path.getmtime(drv), os.path.getmtime(os.path.abspath(__file__))):
        work.append((base + ["-c", drv, "-o", drv_obj], drv_obj, drv_obj + ".log"))
    jobs = jobs or max(1, min(len(work), os.cpu_count() or 4))
    failed = []
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for obj, rc, out in ex.map(_compile, work):
            if rc != 0:
                failed.append((obj, out))
            elif not quiet:
                print("built", os.path.relpath(obj, HERE))
    if failed:
        for obj, out in failed:
            print("FAILED", obj, "\n", "\n".join(l for l in out.splitlines() if "error" in l)[:2000],
                  file=sys.stderr)
        raise RuntimeError("reference build failed (%d files)" % len(failed))
    if work or not os.path.exists(LIB):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + [
            "-lcublas", "-lcufft", "-lcusparse", "-lcudart"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link of libgbref.so failed:\n" + r.stdout[-4000:])
        if not quiet:
            print("linked", os.path.relpath(LIB, HERE))
    return LIB


def build_if_present(reference=None, quiet=True):
    """Build when the reference sources are present; otherwise leave any
    prebuilt library as it is.  Returns the library path or None."""
    reference = reference or os.environ.get("GB_REFERENCE_ROOT", "/root/reference")
    if not os.path.isdir(os.path.join(reference, "toolboxes/nfft/gpu")):
        return LIB if os.path.exists(LIB) else None
    return build(reference, quiet=quiet)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", default=os.environ.get("GB_REFERENCE_ROOT", "/root/reference"))
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.reference, a.jobs, a.force)


if __name__ == "__main__":
    main()
