"""GPU test of gb_nufft_convolve_nc2c_noalloc, the gridding entry point that
allocates no device memory (for callers that cannot call cudaMalloc: host
callbacks, real-time threads with a fixed budget, foreign allocators).  It is called through the C ABI and must reproduce the regular
entry point (gb_nufft_convolve, GB_CONV_NC2C) on two calls in a row, with
heavily loaded tiles so that the split-tile scratch is exercised.

This file is collected last on purpose: a failure here leaves every other
test already run.  It must pass alone in a fresh process and after the rest.
"""
import ctypes

import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from tests.helpers import PARITY_TOL, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402
from gadgetron_b200._lib import lib  # noqa: E402


def _noalloc(plan, samples, grid, accumulate, nb):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.gb_nufft_convolve_nc2c_noalloc(plan._h, ctypes.c_void_p(samples.data_ptr()),
                                              ctypes.c_void_p(grid.data_ptr()), int(accumulate), nb, stream)


def test_noalloc_gridding_matches_regular_entry_point(cuda):
    # Dense radial centre: 192 spokes through a 256x256 grid of 16x16 tiles,
    # so the central tiles' lists are split over several CTAs.
    N, mos, W, C = (128, 128), (256, 256), 5.5, 8
    traj = S.radial_golden_angle_2d(192, 256)
    M = traj.shape[0]
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(cuda))
    rng = np.random.default_rng(0)
    ref = torch.empty((C, 1, 256, 256), dtype=torch.complex64, device=cuda)
    out = torch.empty_like(ref)
    for call in range(2):
        y = torch.from_numpy((rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M)))
                             .astype(np.complex64)).to(cuda)
        plan.convolve(y, ref, gb.NFFT_conv_mode.NC2C)
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert _noalloc(plan, y, out, False, C) == 0, lib.gb_last_error_message()
        torch.cuda.synchronize()
        if call == 1:
            # after the first call's set-up, a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= PARITY_TOL
    # accumulate mode adds onto the output like the regular entry point
    assert _noalloc(plan, y, out, True, C) == 0
    plan.convolve(y, ref, gb.NFFT_conv_mode.NC2C, accumulate=True)
    plan.convolve(y, ref, gb.NFFT_conv_mode.NC2C, accumulate=True)
    ref_once = torch.empty_like(ref)
    plan.convolve(y, ref_once, gb.NFFT_conv_mode.NC2C)
    assert rel_l2(out.cpu().numpy(), 2 * ref_once.cpu().numpy()) <= PARITY_TOL


def test_noalloc_rejects_oversize_and_unprepared(cuda):
    N, mos, W = (64, 64), (128, 128), 5.5
    traj = S.radial_golden_angle_2d(128, 128)
    M = traj.shape[0]
    plan = gb.NFFT.make_plan(N, mos, W)
    y = torch.zeros((1, M), dtype=torch.complex64, device=cuda)
    g = torch.zeros((1, 1, 128, 128), dtype=torch.complex64, device=cuda)
    assert _noalloc(plan, y, g, False, 1) == 3          # not preprocessed
    plan.preprocess(torch.from_numpy(traj).to(cuda))
    nb = 8192   # split scratch = slots x 8192 batches x 256 cells x 8 B, far above 16 MiB
    y = torch.zeros((nb, M), dtype=torch.complex64, device=cuda)
    g = torch.zeros((nb, 1, 128, 128), dtype=torch.complex64, device=cuda)
    assert _noalloc(plan, y, g, False, nb) == 1
    assert b"scratch" in lib.gb_last_error_message()
