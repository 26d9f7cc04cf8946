"""The C++ host interface (include/gadgetron_b200.hpp) compiles and links
against the library (CPU), and on the GPU gives the same results as the
Python binding of the same C ABI."""
import os
import subprocess

import numpy as np
import pytest

from tests.cpp_build import build_driver


def test_cpp_driver_builds(tmp_path):
    exe = build_driver(str(tmp_path / "driver"))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_driver_matches_python(cuda, tmp_path):
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200 import synthetic as S
    N, mos, W, C = 64, 128, 5.5, 4
    traj = S.radial_golden_angle_2d(32, 128)
    M = traj.shape[0]
    sq = np.sqrt(S.ramp_dcw(traj)).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    img = S.ellipse_phantom((N, N), 10, 0)[None]
    rng = np.random.default_rng(0)
    data = (rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))).astype(np.complex64)
    for name, arr in [("traj.f32", traj), ("sqrt_dcw.f32", sq), ("csm.c64", csm), ("image.c64", img),
                      ("data.c64", data)]:
        arr.tofile(str(tmp_path / name))
    exe = build_driver(str(tmp_path / "driver"))
    r = subprocess.run([exe, str(tmp_path), str(N), str(mos), str(W), str(C), str(M), "5"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "iterations 5" in r.stdout and "caught:" in r.stdout
    y_cpp = np.fromfile(str(tmp_path / "y_cpp.c64"), np.complex64).reshape(C, M)
    x_cpp = np.fromfile(str(tmp_path / "x_cpp.c64"), np.complex64).reshape(1, N, N)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(torch.from_numpy(csm).to(cuda))
    E.set_dcw(torch.from_numpy(sq).to(cuda))
    E.preprocess(torch.from_numpy(traj).to(cuda))
    y = torch.empty((C, M), dtype=torch.complex64, device=cuda)
    E.mult_M(torch.from_numpy(img).to(cuda), y)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(5)
    cg.set_tc_tolerance(0.0)
    x = cg.solve(torch.from_numpy(data).to(cuda))
    assert np.array_equal(y.cpu().numpy(), y_cpp)
    assert np.array_equal(x.cpu().numpy(), x_cpp)
