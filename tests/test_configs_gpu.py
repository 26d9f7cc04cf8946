"""GPU parity at the parameters of every benchmark configuration that the
other files do not already cover, against the CPU oracle (itself pinned to
the reference's own outputs in tests/test_ref_parity_gpu.py):

* 2D and 3D NUFFT at alpha 1.5 / W 4 (3D kooshball 64 -> 96, 2D 64 -> 96);
* the variable-density spiral at alpha 1.25 / W 4 (128 -> 160) with
  compensated in-bin accumulation, and the CG-SENSE solve on it with outer
  iterative refinement (3 refinements x 8 iterations);
* the batched uneven multi-frame CG-SENSE with 12 coils at alpha 2, W 5.5,
  frame sizes 13 + (f*37 mod 77) spokes, autotuned tiling, graph capture;
* the trajectory gradient against central finite differences at alpha 1.5,
  W 4 in 2D and 3D.
Tolerances: relative L2 <= 1e-5 for the NUFFT (PARITY_TOL), <= 1e-4 for CG
iterates (FP32 operator, FP64 reductions, against an FP64 oracle CG), 1e-3
relative for the finite-difference gradient.
"""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O
from tests.helpers import PARITY_TOL, kooshball_case, radial_case, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402
from tests.test_autograd_gpu import FD_TOL, _fd_check  # noqa: E402

CG_TOL = 1e-4


def _fwd_adj(case, flags=0):
    dev = torch.device("cuda:0")
    D = len(case["N"])
    plan = gb.NFFT.make_plan(case["N"], case["mos"], case["W"], flags=flags)
    plan.preprocess(torch.from_numpy(case["traj"]).to(dev))
    orc = O.OraclePlan(case["N"], case["mos"], case["W"])
    orc.preprocess(case["traj"].reshape(1, -1, D))
    x = torch.from_numpy(case["img"]).to(dev)
    dcw = torch.from_numpy(case["dcw"]).to(dev)
    y = torch.empty((case["batches"], case["M"]), dtype=torch.complex64, device=dev)
    plan.compute(x, y, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
    ref = orc.forward_c2nc(case["img"])
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    back = torch.empty_like(x)
    plan.compute(y, back, dcw, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    assert rel_l2(back.cpu().numpy(), orc.backwards_nc2c(ref, case["dcw"].reshape(1, -1))) <= PARITY_TOL


def test_3d_alpha_1_5_w4():
    case = kooshball_case(N=64, alpha=1.5, W=4.0, spokes=600, samples=64, batches=2, seed=21)
    assert case["mos"] == (96, 96, 96)
    _fwd_adj(case)


def test_2d_alpha_1_5_w4():
    case = radial_case(N=64, alpha=1.5, W=4.0, spokes=48, samples=128, batches=3, seed=22)
    assert case["mos"] == (96, 96)
    _fwd_adj(case)


def _spiral_case(coils=8, seed=23):
    N, mos, W = (128, 128), (160, 160), 4.0
    traj = S.spiral_archimedean_2d(24, 1024, 128)
    dcw = S.ramp_dcw(traj)
    img = S.gaussian_image((coils, 1, 128, 128), seed)
    return dict(N=N, mos=mos, W=W, traj=traj, dcw=dcw, img=img, M=traj.shape[0], batches=coils)


@pytest.mark.parametrize("compensated", [False, True])
def test_spiral_alpha_1_25_w4(compensated):
    case = _spiral_case()
    _fwd_adj(case, flags=gb.FLAG_COMPENSATED if compensated else 0)


def test_spiral_cg_sense_iterative_refinement():
    """3 refinements x 8 CG iterations on the spiral with compensated
    gridding, against the oracle's FP64 refinement loop; the refined solve
    has a smaller normal-equation residual than one 8-iteration solve."""
    dev = torch.device("cuda:0")
    N, mos, W, C = (128, 128), (160, 160), 4.0, 8
    traj = S.spiral_archimedean_2d(24, 1024, 128)
    sq = np.sqrt(S.ramp_dcw(traj)).astype(np.float32)
    csm = S.gaussian_bump_csm((128, 128), C)
    ph = S.ellipse_phantom((128, 128), 20, 24)[None]
    plan = O.OraclePlan(N, mos, W)
    plan.preprocess(traj[None])
    orc = O.OracleSense(plan, csm, sq[None])
    d = orc.mult_M(ph)
    rng = np.random.default_rng(25)
    d = (d + 0.01 * np.sqrt(np.mean(np.abs(d) ** 2)) * (rng.standard_normal(d.shape) +
                                                        1j * rng.standard_normal(d.shape)) / np.sqrt(2)
         ).astype(np.complex64)
    E = gb.cuNonCartesianSenseOperator(2, flags=gb.FLAG_COMPENSATED)
    E.setup(N, mos, W)
    E.set_csm(torch.from_numpy(csm).to(dev))
    E.set_dcw(torch.from_numpy(sq).to(dev))
    E.preprocess(torch.from_numpy(traj).to(dev))
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(8)
    cg.set_tc_tolerance(0.0)
    cg.set_refinements(3)
    d_t = torch.from_numpy(d.reshape(C, -1)).to(dev)
    x = cg.solve(d_t).cpu().numpy()
    xr = O.cg_solve_refined(orc, d, iterations=8, refinements=3)
    assert rel_l2(x, xr) <= CG_TOL
    cg.set_refinements(1)
    x1 = cg.solve(d_t).cpu().numpy()
    rhs = orc.mult_MH(d)
    res = lambda v: np.linalg.norm(orc.mult_MH_M(v.astype(np.complex128)) - rhs)
    assert res(x) < res(x1)
    assert E.get_plan().device_errors() == 0


def test_batched_uneven_12_coils_autotuned():
    """Uneven frames of 13 + (f*37 mod 77) golden-angle spokes, 12 coils,
    alpha 2 / W 5.5, all frames in one operator with autotuned tiling and the
    CG iteration captured in a graph, against one oracle solve per frame."""
    dev = torch.device("cuda:0")
    N, mos, W, C, F, iters = 64, 128, 5.5, 12, 6, 8
    spokes = [13 + (f * 37) % 77 for f in range(F)]
    trajs = [S.radial_golden_angle_2d(s, 96, profile_offset=sum(spokes[:f])) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    sq = np.concatenate([np.sqrt(S.ramp_dcw(t)) for t in trajs]).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    rng = np.random.default_rng(26)
    base = S.ellipse_phantom((N, N), 12, 27)
    ph = np.stack([base * rng.uniform(0.9, 1.1) for _ in range(F)], 0).astype(np.complex64)
    d = np.zeros((C, offs[-1]), np.complex64)
    ops = []
    for f in range(F):
        P = O.OraclePlan((N, N), (mos, mos), W)
        P.preprocess(trajs[f][None])
        Ef = O.OracleSense(P, csm, sq[offs[f]:offs[f + 1]][None])
        d[:, offs[f]:offs[f + 1]] = Ef.mult_M(ph[f:f + 1]).reshape(C, -1)
        ops.append(Ef)
    E = gb.cuNonCartesianSenseOperator(2, flags=gb.FLAG_AUTOTUNE)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(torch.from_numpy(csm).to(dev))
    E.set_dcw(torch.from_numpy(sq).to(dev))
    E.preprocess(torch.from_numpy(traj).to(dev), frame_offsets=offs)
    tile, group = E.get_plan().get_tiling()
    assert group in (4, 8, 12, 16) and all(t > 0 for t in tile)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(iters)
    cg.set_tc_tolerance(0.0)
    cg.set_frame_independent(True)
    cg.set_use_graph(True)
    xb = cg.solve(torch.from_numpy(d).to(dev)).cpu().numpy()
    for f in range(F):
        xr = O.cg_solve(ops[f], d[:, offs[f]:offs[f + 1]][:, None, :], iterations=iters, tc_tolerance=0.0)
        assert rel_l2(xb[f], xr[0]) <= CG_TOL, f
    assert E.get_plan().device_errors() == 0


def test_traj_grad_fd_2d_alpha_1_5_w4():
    traj = S.radial_golden_angle_2d(48, 128)
    err, frac = _fd_check(traj, (64, 64), (96, 96), 4.0, nb=2, seed=28)
    assert frac > 0.5
    assert err <= FD_TOL, err


def test_traj_grad_fd_3d_alpha_1_5_w4():
    traj = S.kooshball_golden_means_3d(400, 64)
    err, frac = _fd_check(traj, (64, 64, 64), (96, 96, 96), 4.0, nb=2, seed=29)
    assert frac > 0.5
    assert err <= FD_TOL, err


def test_batched_many_frames_deep_launch_schedules():
    """48 uneven frames of 64^2 (mos 128, 64 tiles a frame): the gridding
    launch of E^H E is more than 8 resident waves deep.  Schedule 1 takes the
    register-staged gridding over the plan's sorted sample layout, schedule 2
    (and the default) the persistent work-queue kernel over the interleaved
    layout (small launches take the per-item warp-specialized kernel,
    covered by every other CG test).  Both give the same images bit for bit;
    frame-independent CG against one oracle solve per frame."""
    dev = torch.device("cuda:0")
    N, mos, W, C, F, iters = 64, 128, 5.5, 8, 48, 6
    spokes = [4 + (f * 5) % 9 for f in range(F)]
    trajs = [S.radial_golden_angle_2d(s, 64, profile_offset=sum(spokes[:f])) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    sq = np.concatenate([np.sqrt(S.ramp_dcw(t)) for t in trajs]).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    base = S.ellipse_phantom((N, N), 8, 41)
    rng = np.random.default_rng(42)
    ph = np.stack([base * rng.uniform(0.9, 1.1) for _ in range(F)], 0).astype(np.complex64)
    d = np.zeros((C, offs[-1]), np.complex64)
    ops = []
    for f in range(F):
        P = O.OraclePlan((N, N), (mos, mos), W)
        P.preprocess(trajs[f][None])
        Ef = O.OracleSense(P, csm, sq[offs[f]:offs[f + 1]][None])
        d[:, offs[f]:offs[f + 1]] = Ef.mult_M(ph[f:f + 1]).reshape(C, -1)
        ops.append(Ef)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(torch.from_numpy(csm).to(dev))
    E.set_dcw(torch.from_numpy(sq).to(dev))
    E.preprocess(torch.from_numpy(traj).to(dev), frame_offsets=offs)
    E.get_plan().set_tiling((16, 16), 8)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(iters)
    cg.set_tc_tolerance(0.0)
    cg.set_frame_independent(True)
    refs = {f: O.cg_solve(ops[f], d[:, offs[f]:offs[f + 1]][:, None, :], iterations=iters, tc_tolerance=0.0)
            for f in range(0, F, 7)}
    sols = {}
    for sched in (1, 2):
        E.get_plan().set_grid_schedule(sched)
        for use_graph in (False, True):
            cg.set_use_graph(use_graph)
            xb = cg.solve(torch.from_numpy(d).to(dev)).cpu().numpy()
            sols[(sched, use_graph)] = xb
            for f, xr in refs.items():
                assert rel_l2(xb[f], xr[0]) <= CG_TOL, (sched, use_graph, f)
    assert np.array_equal(sols[(1, True)], sols[(2, True)])
    assert np.array_equal(sols[(1, False)], sols[(2, False)])
    assert E.get_plan().device_errors() == 0
