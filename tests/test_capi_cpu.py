"""CPU checks of the C ABI (no GPU needed): the library loads, exports every
symbol include/gadgetron_b200.h declares, and rejects invalid arguments with
the documented status codes before touching the device (the reference throws
std::runtime_error for the same conditions,
toolboxes/nfft/gpu/cuGriddingConvolution.cu:56-80)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gadgetron_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"GB_API\s+[^;{]*?\b(gb_\w+)\s*\(", txt)))


def test_library_exports_header_symbols():
    from gadgetron_b200 import _lib
    syms = header_symbols()
    assert len(syms) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(gb_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == syms
    for s in syms:
        assert hasattr(_lib.lib, s)


def test_build_targets_sm100a_only():
    import importlib.util
    spec = importlib.util.spec_from_file_location("_gb_build", os.path.join(ROOT, "gadgetron_b200", "build.py"))
    B = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(B)
    flags = " ".join(B.ARCH + B.CFLAGS)
    assert set(re.findall(r"arch=(\S+?),code=(\S+)", flags)) == {("compute_100a", "sm_100a")}


def _u64(v):
    return (ctypes.c_uint64 * len(v))(*v)


def test_invalid_arguments_rejected_without_device():
    from gadgetron_b200 import _lib
    L = _lib.lib
    h = ctypes.c_void_p()
    # kernel width below 1.8
    assert L.gb_nufft_plan_create(2, _u64([64, 64]), _u64([128, 128]), ctypes.c_float(1.5), 0, ctypes.byref(h)) == 1
    assert b"1.8" in L.gb_last_error_message()
    # not a multiple of 32
    assert L.gb_nufft_plan_create(2, _u64([48, 48]), _u64([96, 100]), ctypes.c_float(5.5), 0, ctypes.byref(h)) == 1
    assert b"multiple of 32" in L.gb_last_error_message()
    # oversampled smaller than matrix
    assert L.gb_nufft_plan_create(2, _u64([64, 64]), _u64([32, 32]), ctypes.c_float(5.5), 0, ctypes.byref(h)) == 1
    # unsupported dimensionality
    assert L.gb_nufft_plan_create(4, _u64([32] * 4), _u64([64] * 4), ctypes.c_float(5.5), 0, ctypes.byref(h)) == 1
    # NULL output handle
    assert L.gb_nufft_plan_create(2, _u64([64, 64]), _u64([128, 128]), ctypes.c_float(5.5), 0, None) == 1
    # NULL plan
    assert L.gb_nufft_compute(None, None, None, None, 0, 1, 0, None) == 1
    assert L.gb_sense_mult_M(None, None, None, 0, None) == 1


def test_cg_host_state_without_device():
    from gadgetron_b200 import _lib
    L = _lib.lib
    s = ctypes.c_void_p()
    assert L.gb_cg_create(ctypes.byref(s)) == 0
    assert L.gb_cg_set_max_iterations(s, 5) == 0
    assert L.gb_cg_set_tc_tolerance(s, ctypes.c_float(0.0)) == 0
    assert L.gb_cg_set_refinements(s, 0) == 1
    # no encoding operator: the reference throws from compute_rhs
    assert L.gb_cg_solve(s, None, None, None, None, None) == 1
    assert b"encoding operator" in L.gb_last_error_message()
    assert L.gb_cg_destroy(s) == 0


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "gadgetron_b200.h"\nint main(void){gb_nufft_plan p=0;(void)p;return 0;}\n')
    for cc in (["gcc", "-std=c99"], ["g++", "-std=c++17", "-x", "c++"]):
        r = subprocess.run(cc + ["-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_product_fails_loudly_without_library(tmp_path):
    """The package has no CPU fallback: without the .so, import fails."""
    code = ("import sys, importlib.util; sys.path.insert(0, %r);"
            "import gadgetron_b200._lib as L" % ROOT)
    env = dict(os.environ)
    r = subprocess.run(["python", "-c", code + "; print(L.LIB_PATH)"], capture_output=True, text=True, env=env)
    assert r.returncode == 0
    # simulate a missing library by pointing the loader at a non-existent path
    code2 = ("import sys, os; sys.path.insert(0, %r); import gadgetron_b200._lib as L;"
             "L.LIB_PATH = '/nonexistent/lib.so';\n"
             "try:\n    L._load()\nexcept ImportError as e:\n    print('IMPORT-ERROR', e)\n" % ROOT)
    r = subprocess.run(["python", "-c", code2], capture_output=True, text=True)
    assert "IMPORT-ERROR" in r.stdout


def test_lazy_conj_views_are_rejected():
    import torch
    from gadgetron_b200.nfft import _check_tensor
    t = torch.zeros(4, dtype=torch.complex64)
    with pytest.raises(ValueError):
        _check_tensor(t.conj(), torch.complex64, "x")
