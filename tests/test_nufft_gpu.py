"""GPU parity of the NUFFT plan (through the C ABI) against the CPU oracle.

Mirrors what the reference's own test of cuNFFT exercises
(test/cuNFFT_test.cpp: BACKWARDS_NC2C on multi-coil radial data) and adds the
value checks it lacks: every compute mode, mult_MH_M, the standalone
convolve/fft/deapodize utilities, uneven frames, accumulation, determinism.
Tolerance: relative L2 <= 1e-5 against the oracle (FP32 vs the reference
algorithm summed in FP64).
"""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O
from tests.helpers import PARITY_TOL, kooshball_case, radial_case, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402


def _plan_and_oracle(case, flags=0, frame_offsets=None):
    dev = torch.device("cuda:0")
    plan = gb.NFFT.make_plan(case["N"], case["mos"], case["W"], flags=flags)
    traj_t = torch.from_numpy(case["traj"]).to(dev)
    if frame_offsets is None:
        plan.preprocess(traj_t, gb.NFFT_prep_mode.ALL, num_frames=case["frames"])
    else:
        plan.preprocess(traj_t, gb.NFFT_prep_mode.ALL, frame_offsets=frame_offsets)
    orc = O.OraclePlan(case["N"], case["mos"], case["W"])
    F = case["frames"]
    orc.preprocess(case["traj"].reshape(F, -1, len(case["N"])))
    return plan, orc, traj_t


@pytest.mark.parametrize("batches", [1, 3, 16])
def test_forward_c2nc_2d(cuda, batches):
    case = radial_case(N=64, spokes=24, samples=128, batches=batches, seed=batches)
    plan, orc, _ = _plan_and_oracle(case)
    x = torch.from_numpy(case["img"]).to(cuda)
    dcw = torch.from_numpy(case["dcw"]).to(cuda)
    y = torch.empty((batches, case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(x, y, dcw, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(case["img"], case["dcw"].reshape(1, -1))
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL


@pytest.mark.parametrize("batches", [1, 5])
def test_backwards_nc2c_2d(cuda, batches):
    case = radial_case(N=64, spokes=24, samples=128, batches=batches, seed=10 + batches)
    plan, orc, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(5)
    y = (rng.standard_normal((batches, case["M"])) + 1j * rng.standard_normal((batches, case["M"]))).astype(np.complex64)
    out = torch.empty((batches, 1, 64, 64), dtype=torch.complex64, device=cuda)
    plan.compute(torch.from_numpy(y).to(cuda), out, torch.from_numpy(case["dcw"]).to(cuda),
                 gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref = orc.backwards_nc2c(y, case["dcw"].reshape(1, -1))
    assert rel_l2(out.cpu().numpy(), ref) <= PARITY_TOL


def test_forwards_nc2c_2d(cuda):
    case = radial_case(N=64, spokes=16, samples=128, batches=2, seed=3)
    plan, orc, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(6)
    y = (rng.standard_normal((2, case["M"])) + 1j * rng.standard_normal((2, case["M"]))).astype(np.complex64)
    out = torch.empty((2, 1, 64, 64), dtype=torch.complex64, device=cuda)
    plan.compute(torch.from_numpy(y).to(cuda), out, None, gb.NFFT_comp_mode.FORWARDS_NC2C)
    ref = orc.forwards_nc2c(y)
    assert rel_l2(out.cpu().numpy(), ref) <= PARITY_TOL


def test_oversampled_image_modes(cuda):
    case = radial_case(N=32, spokes=16, samples=64, batches=2, seed=4)
    plan, orc, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(7)
    xo = (rng.standard_normal((2, 1, 64, 64)) + 1j * rng.standard_normal((2, 1, 64, 64))).astype(np.complex64)
    y = torch.empty((2, case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(torch.from_numpy(xo).to(cuda), y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(xo)
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty((2, 1, 64, 64), dtype=torch.complex64, device=cuda)
    plan.compute(y, back, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref2 = orc.backwards_nc2c(y.cpu().numpy(), oversampled_out=True)
    assert rel_l2(back.cpu().numpy(), ref2) <= PARITY_TOL
    # image-sized call after an oversampled one (padded buffer must be re-zeroed)
    x = torch.from_numpy(case["img"]).to(cuda)
    y2 = torch.empty((2, case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(x, y2, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref3 = orc.forward_c2nc(x.cpu().numpy())
    assert rel_l2(y2.cpu().numpy(), ref3) <= PARITY_TOL


def test_mult_MH_M_2d(cuda):
    case = radial_case(N=64, spokes=32, samples=128, batches=4, seed=8)
    plan, orc, _ = _plan_and_oracle(case)
    x = torch.from_numpy(case["img"]).to(cuda)
    out = torch.empty_like(x)
    dcw = torch.from_numpy(case["dcw"]).to(cuda)
    plan.mult_MH_M(x, out, dcw)
    ref = orc.mult_MH_M(case["img"], case["dcw"].reshape(1, -1))
    assert rel_l2(out.cpu().numpy(), ref) <= PARITY_TOL


def test_multiframe_equal(cuda):
    case = radial_case(N=32, spokes=8, samples=64, frames=3, batches=2, seed=9)
    plan, orc, _ = _plan_and_oracle(case)
    x = torch.from_numpy(case["img"]).to(cuda)
    y = torch.empty((2, 3 * case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(case["img"])
    assert rel_l2(y.cpu().numpy(), ref.reshape(2, -1)) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref2 = orc.backwards_nc2c(ref)
    assert rel_l2(back.cpu().numpy(), ref2) <= PARITY_TOL


def test_uneven_frames_match_per_frame(cuda):
    """Frames with different sample counts in one plan equal per-frame plans."""
    from gadgetron_b200 import synthetic as S
    N, mos, W = (32, 32), (64, 64), 5.5
    spokes = [5, 9, 3]
    trajs = [S.radial_golden_angle_2d(s, 64, profile_offset=7 * f) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    C = 2
    rng = np.random.default_rng(11)
    img = (rng.standard_normal((C, 3, 32, 32)) + 1j * rng.standard_normal((C, 3, 32, 32))).astype(np.complex64)
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(cuda), frame_offsets=offs)
    y = torch.empty((C, offs[-1]), dtype=torch.complex64, device=cuda)
    plan.compute(torch.from_numpy(img).to(cuda), y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    back = torch.empty((C, 3, 32, 32), dtype=torch.complex64, device=cuda)
    plan.compute(y, back, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    yc, bc = y.cpu().numpy(), back.cpu().numpy()
    for f in range(3):
        orc = O.OraclePlan(N, mos, W)
        orc.preprocess(trajs[f][None])
        ref = orc.forward_c2nc(img[:, f:f + 1])
        assert rel_l2(yc[:, offs[f]:offs[f + 1]], ref.reshape(C, -1)) <= PARITY_TOL
        refb = orc.backwards_nc2c(yc[:, offs[f]:offs[f + 1]])
        assert rel_l2(bc[:, f], refb.reshape(C, 32, 32)) <= PARITY_TOL


def test_3d_forward_adjoint(cuda):
    case = kooshball_case(N=64, spokes=300, samples=64, batches=3, seed=12)
    plan, orc, _ = _plan_and_oracle(case)
    x = torch.from_numpy(case["img"]).to(cuda)
    dcw = torch.from_numpy(case["dcw"]).to(cuda)
    y = torch.empty((3, case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(x, y, dcw, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(case["img"], case["dcw"].reshape(1, -1))
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, dcw, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref2 = orc.backwards_nc2c(ref, case["dcw"].reshape(1, -1))
    assert rel_l2(back.cpu().numpy(), ref2) <= PARITY_TOL


# Oversampled sizes covering every transform length of the project-written
# FFT passes (16 * n2, n2 in 2, 4, 6, 8, 10, 12, 16, 20, 24, 32, 40) on
# non-square grids, and one size they do not cover (224 = 16 * 14: the plan
# then uses cuFFT for every pass).
@pytest.mark.parametrize("N,mos", [((32, 64), (96, 160)), ((64, 32), (320, 64)), ((32, 32), (224, 128)),
                                   ((64, 64), (384, 640)), ((32, 96), (128, 192)), ((128, 32), (256, 32)),
                                   ((64, 128), (512, 256))])
def test_fft_lengths_2d(cuda, N, mos):
    W, batches = 4.0, 2
    traj = S.radial_golden_angle_2d(24, 96)
    dcw = S.ramp_dcw(traj)
    img = S.gaussian_image((batches, 1, N[1], N[0]), 31)
    dev = torch.device("cuda:0")
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(dev), gb.NFFT_prep_mode.ALL)
    orc = O.OraclePlan(N, mos, W)
    orc.preprocess(traj.reshape(1, -1, 2))
    x = torch.from_numpy(img).to(dev)
    y = torch.empty((batches, traj.shape[0]), dtype=torch.complex64, device=dev)
    plan.compute(x, y, torch.from_numpy(dcw).to(dev), gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(img, dcw.reshape(1, -1))
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, torch.from_numpy(dcw).to(dev), gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref2 = orc.backwards_nc2c(ref, dcw.reshape(1, -1))
    assert rel_l2(back.cpu().numpy(), ref2) <= PARITY_TOL


def test_fft_lengths_3d(cuda):
    N, mos, W = (32, 32, 32), (64, 96, 160), 4.0
    traj = S.kooshball_golden_means_3d(150, 48)
    dcw = S.ramp_dcw(traj)
    img = S.gaussian_image((2, 1, 32, 32, 32), 32)
    dev = torch.device("cuda:0")
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(dev), gb.NFFT_prep_mode.ALL)
    orc = O.OraclePlan(N, mos, W)
    orc.preprocess(traj.reshape(1, -1, 3))
    x = torch.from_numpy(img).to(dev)
    y = torch.empty((2, traj.shape[0]), dtype=torch.complex64, device=dev)
    plan.compute(x, y, torch.from_numpy(dcw).to(dev), gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(img, dcw.reshape(1, -1))
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, torch.from_numpy(dcw).to(dev), gb.NFFT_comp_mode.BACKWARDS_NC2C)
    ref2 = orc.backwards_nc2c(ref, dcw.reshape(1, -1))
    assert rel_l2(back.cpu().numpy(), ref2) <= PARITY_TOL


def test_convolve_and_accumulate(cuda):
    case = radial_case(N=32, spokes=16, samples=64, batches=2, seed=13)
    plan, orc, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(14)
    grid = (rng.standard_normal((2, 1, 64, 64)) + 1j * rng.standard_normal((2, 1, 64, 64))).astype(np.complex64)
    y = torch.empty((2, case["M"]), dtype=torch.complex64, device=cuda)
    plan.convolve(torch.from_numpy(grid).to(cuda), y, gb.NFFT_conv_mode.C2NC)
    ref = orc.convolve_c2nc(grid)
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    plan.convolve(torch.from_numpy(grid).to(cuda), y, gb.NFFT_conv_mode.C2NC, accumulate=True)
    assert rel_l2(y.cpu().numpy(), 2 * ref) <= PARITY_TOL
    g = torch.empty((2, 1, 64, 64), dtype=torch.complex64, device=cuda)
    plan.convolve(y, g, gb.NFFT_conv_mode.NC2C)
    refg = orc.convolve_nc2c(2 * ref)
    assert rel_l2(g.cpu().numpy(), refg) <= PARITY_TOL
    plan.convolve(y, g, gb.NFFT_conv_mode.NC2C, accumulate=True)
    assert rel_l2(g.cpu().numpy(), 2 * refg) <= PARITY_TOL


def test_fft_and_deapodize_utilities(cuda):
    case = radial_case(N=32, spokes=8, samples=64, batches=1, seed=15)
    plan, orc, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(16)
    a = (rng.standard_normal((3, 1, 64, 64)) + 1j * rng.standard_normal((3, 1, 64, 64))).astype(np.complex64)
    t = torch.from_numpy(a).to(cuda)
    plan.fft(t, gb.NFFT_fft_mode.FORWARDS)
    assert rel_l2(t.cpu().numpy(), O.centred_fft(a, 2, True)) <= PARITY_TOL
    plan.fft(t, gb.NFFT_fft_mode.BACKWARDS, do_scale=False)
    assert rel_l2(t.cpu().numpy(), O.centred_fft(O.centred_fft(a, 2, True), 2, False, False)) <= PARITY_TOL
    t2 = torch.from_numpy(a).to(cuda)
    plan.deapodize(t2)
    assert rel_l2(t2.cpu().numpy(), orc.deapodize(a)) <= PARITY_TOL


def test_determinism(cuda):
    case = radial_case(N=64, spokes=64, samples=128, batches=4, seed=17)
    plan, _, _ = _plan_and_oracle(case)
    rng = np.random.default_rng(18)
    y = torch.from_numpy((rng.standard_normal((4, case["M"])) +
                          1j * rng.standard_normal((4, case["M"]))).astype(np.complex64)).to(cuda)
    a = torch.empty((4, 1, 64, 64), dtype=torch.complex64, device=cuda)
    b = torch.empty_like(a)
    plan.compute(y, a, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    plan.compute(y, b, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    assert torch.equal(a, b)


def test_repeated_preprocess_replays_recorded_segments(cuda):
    """Preprocess records its two device segments as graphs the second time
    the same shapes arrive on the same buffers and replays them after that.
    A trajectory changed in place between calls (same buffer, new values, so
    every later call replays) must give the results of a fresh plan; an
    out-of-range trajectory is still reported on a replay; a trajectory of
    another length re-runs eagerly."""
    case = radial_case(N=64, spokes=24, samples=128, batches=2, seed=51)
    dev = torch.device("cuda:0")
    other = S.radial_golden_angle_2d(24, 128, profile_offset=977).astype(np.float32)
    traj_t = torch.from_numpy(case["traj"]).to(dev)
    plan = gb.NFFT.make_plan(case["N"], case["mos"], case["W"])
    x = torch.from_numpy(case["img"]).to(dev)
    for rep in range(4):   # eager, recorded, replayed, replayed
        src = case["traj"] if rep % 2 == 0 else other
        traj_t.copy_(torch.from_numpy(src))
        plan.preprocess(traj_t)
        y = torch.empty((case["batches"], case["M"]), dtype=torch.complex64, device=dev)
        plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
        fresh = gb.NFFT.make_plan(case["N"], case["mos"], case["W"])
        fresh.preprocess(torch.from_numpy(src).to(dev))
        y2 = torch.empty_like(y)
        fresh.compute(x, y2, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
        assert torch.equal(y, y2), rep
        back = torch.empty_like(x)
        plan.compute(y, back, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
        back2 = torch.empty_like(x)
        fresh.compute(y2, back2, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
        assert torch.equal(back, back2), rep
    bad = case["traj"].copy()
    bad[5, 0] = 0.75
    traj_t.copy_(torch.from_numpy(bad))
    with pytest.raises(RuntimeError):
        plan.preprocess(traj_t)
    short = torch.from_numpy(case["traj"][: case["M"] // 2].copy()).to(dev)
    plan.preprocess(short)
    orc = O.OraclePlan(case["N"], case["mos"], case["W"])
    orc.preprocess(case["traj"][: case["M"] // 2].reshape(1, -1, 2))
    y = torch.empty((case["batches"], case["M"] // 2), dtype=torch.complex64, device=dev)
    plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    assert rel_l2(y.cpu().numpy(), orc.forward_c2nc(case["img"])) <= PARITY_TOL


def test_error_paths(cuda):
    plan = gb.NFFT.make_plan((32, 32), (64, 64), 5.5)
    x = torch.zeros((1, 1, 32, 32), dtype=torch.complex64, device=cuda)
    y = torch.zeros((1, 64), dtype=torch.complex64, device=cuda)
    with pytest.raises(gb.NotPreprocessedError):
        plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    bad = torch.full((64, 2), 0.6, dtype=torch.float32, device=cuda)
    with pytest.raises(gb.TrajectoryRangeError):
        plan.preprocess(bad)
    with pytest.raises(gb.GadgetronB200Error):
        gb.NFFT.make_plan((30, 30), (64, 64), 5.5)
    with pytest.raises(gb.GadgetronB200Error):
        gb.NFFT.make_plan((32, 32), (64, 64), 1.5)


def test_autotune_keeps_parity(cuda):
    case = radial_case(N=64, spokes=48, samples=128, batches=8, seed=21)
    plan, orc, _ = _plan_and_oracle(case)
    before = plan.get_tiling()
    plan.autotune(8)
    tile, cg = plan.get_tiling()
    assert cg in (4, 8, 16) and len(tile) == 2
    x = torch.from_numpy(case["img"]).to(cuda)
    y = torch.empty((8, case["M"]), dtype=torch.complex64, device=cuda)
    plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(case["img"])
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, None, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    assert rel_l2(back.cpu().numpy(), orc.backwards_nc2c(ref)) <= PARITY_TOL
    # an explicit tiling re-bins the preprocessed trajectory
    plan.set_tiling((32, 16), 8)
    assert plan.get_tiling() == ((32, 16), 8)
    plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    del before


def test_time_normal_convolutions_diagnostic(cuda):
    """The diagnostic timing of E^H E's two convolutions returns positive
    times and leaves the plan usable (its workspaces are scratch)."""
    case = radial_case(N=64, spokes=32, samples=128, batches=8, seed=19)
    plan, orc, _ = _plan_and_oracle(case)
    dcw = torch.from_numpy(case["dcw"]).to(cuda)
    flush = torch.empty(64 * 1024 * 1024 // 4, dtype=torch.float32, device=cuda)
    tg, td = plan.time_normal_convolutions(8, dcw, reps=3, flush=flush)
    assert 0.0 < tg < 100.0 and 0.0 < td < 100.0
    x = torch.from_numpy(case["img"]).to(cuda)
    out = torch.empty_like(x)
    plan.mult_MH_M(x, out, dcw)
    assert rel_l2(out.cpu().numpy(), orc.mult_MH_M(case["img"], case["dcw"].reshape(1, -1))) <= PARITY_TOL
