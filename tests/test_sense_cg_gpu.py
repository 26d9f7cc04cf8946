"""GPU parity of the non-Cartesian SENSE operator and the CG-SENSE solver
against the CPU oracle (cuNonCartesianSenseOperator.cu:14-62 and
cgSolver.h:105-390 restated in oracle/oracle.py)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from gadgetron_b200 import synthetic as S
from tests.helpers import PARITY_TOL, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402


def sense_case(N=64, alpha=2.0, W=5.5, spokes=48, samples=128, coils=8, frames=1, seed=0):
    mos = int(round(N * alpha))
    traj = np.concatenate([S.radial_golden_angle_2d(spokes, samples, profile_offset=f * spokes)
                           for f in range(frames)], 0)
    dcw = np.concatenate([S.ramp_dcw(traj[f * spokes * samples:(f + 1) * spokes * samples])
                          for f in range(frames)], 0)
    sq = np.sqrt(dcw).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), coils)
    ph = np.stack([S.ellipse_phantom((N, N), 20, seed + f) for f in range(frames)], 0)
    return dict(N=(N, N), mos=(mos, mos), W=W, traj=traj, sqrt_dcw=sq, csm=csm, phantom=ph, frames=frames,
                M=spokes * samples, coils=coils)


def make_ops(case, cuda, flags=0):
    E = gb.cuNonCartesianSenseOperator(2, flags=flags)
    E.setup(case["N"], case["mos"], case["W"])
    E.set_csm(torch.from_numpy(case["csm"]).to(cuda))
    E.set_dcw(torch.from_numpy(case["sqrt_dcw"]).to(cuda))
    E.preprocess(torch.from_numpy(case["traj"]).to(cuda), num_frames=case["frames"])
    plan = O.OraclePlan(case["N"], case["mos"], case["W"])
    plan.preprocess(case["traj"].reshape(case["frames"], -1, 2))
    orc = O.OracleSense(plan, case["csm"], case["sqrt_dcw"].reshape(case["frames"], -1))
    return E, orc


def test_sense_mult_M_MH(cuda):
    case = sense_case(coils=8, seed=1)
    E, orc = make_ops(case, cuda)
    x = torch.from_numpy(case["phantom"]).to(cuda)
    y = torch.empty((8, case["M"]), dtype=torch.complex64, device=cuda)
    E.mult_M(x, y)
    ref = orc.mult_M(case["phantom"])
    assert rel_l2(y.cpu().numpy(), ref) <= PARITY_TOL
    xb = torch.empty_like(x)
    E.mult_MH(y, xb)
    refb = orc.mult_MH(ref)
    assert rel_l2(xb.cpu().numpy(), refb) <= PARITY_TOL
    E.mult_MH(y, xb, accumulate=True)
    assert rel_l2(xb.cpu().numpy(), 2 * refb) <= PARITY_TOL
    xn = torch.empty_like(x)
    E.mult_MH_M(x, xn)
    assert rel_l2(xn.cpu().numpy(), orc.mult_MH_M(case["phantom"])) <= PARITY_TOL


@pytest.mark.parametrize("coils", [12, 24])
def test_sense_coil_groups_of_12(cuda, coils):
    """Coil counts that are multiples of 12 degrid in groups of 12 (no empty
    coil slots); forward and normal operator against the oracle."""
    case = sense_case(N=32, spokes=24, samples=64, coils=coils, seed=11)
    E, orc = make_ops(case, cuda)
    x = torch.from_numpy(case["phantom"]).to(cuda)
    y = torch.empty((coils, case["M"]), dtype=torch.complex64, device=cuda)
    E.mult_M(x, y)
    assert rel_l2(y.cpu().numpy(), orc.mult_M(case["phantom"])) <= PARITY_TOL
    xn = torch.empty_like(x)
    E.mult_MH_M(x, xn)
    assert rel_l2(xn.cpu().numpy(), orc.mult_MH_M(case["phantom"])) <= PARITY_TOL


def test_sense_multiframe(cuda):
    case = sense_case(N=32, spokes=16, samples=64, coils=4, frames=3, seed=2)
    E, orc = make_ops(case, cuda)
    x = torch.from_numpy(case["phantom"]).to(cuda)
    y = torch.empty((4, 3 * case["M"]), dtype=torch.complex64, device=cuda)
    E.mult_M(x, y)
    ref = orc.mult_M(case["phantom"])
    assert rel_l2(y.cpu().numpy(), ref.reshape(4, -1)) <= PARITY_TOL
    xb = torch.empty_like(x)
    E.mult_MH(y, xb)
    assert rel_l2(xb.cpu().numpy(), orc.mult_MH(ref)) <= PARITY_TOL


@pytest.mark.parametrize("use_graph", [False, True])
def test_cg_sense_matches_oracle(cuda, use_graph):
    case = sense_case(coils=8, seed=3)
    E, orc = make_ops(case, cuda)
    d_ref = orc.mult_M(case["phantom"])
    rng = np.random.default_rng(4)
    noise = 0.01 * np.sqrt(np.mean(np.abs(d_ref) ** 2)) * (rng.standard_normal(d_ref.shape) +
                                                          1j * rng.standard_normal(d_ref.shape)) / np.sqrt(2)
    d = (d_ref + noise).astype(np.complex64)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(10)
    cg.set_tc_tolerance(0.0)
    cg.set_use_graph(use_graph)
    x = cg.solve(torch.from_numpy(d.reshape(8, -1)).to(cuda))
    hist = []
    xr = O.cg_solve(orc, d, iterations=10, tc_tolerance=0.0, history=hist)
    assert cg.last_iterations == 10
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4
    h = cg.residual_history[:10].cpu().numpy()
    assert np.allclose(h, hist, rtol=1e-3)
    if use_graph:
        x2 = cg.solve(torch.from_numpy(d.reshape(8, -1)).to(cuda))
        assert torch.equal(x, x2)
    # no bounded wait (bulk-copy mbarrier, fused-tail grid barrier) ran out
    assert E.get_plan().device_errors() == 0


def test_cg_early_stop_and_x0(cuda):
    case = sense_case(coils=4, seed=5)
    E, orc = make_ops(case, cuda)
    d = orc.mult_M(case["phantom"]).astype(np.complex64)
    dt = torch.from_numpy(d.reshape(4, -1)).to(cuda)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(30)
    cg.set_tc_tolerance(1e-3)
    x = cg.solve(dt)
    hist = []
    xr = O.cg_solve(orc, d, iterations=30, tc_tolerance=1e-3, history=hist)
    assert cg.last_iterations == len(hist)
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4
    x0 = torch.from_numpy(case["phantom"] * 0.5).to(cuda)
    cg.set_x0(x0)
    cg.set_tc_tolerance(0.0)
    cg.set_max_iterations(5)
    x = cg.solve(dt)
    xr = O.cg_solve(orc, d, iterations=5, tc_tolerance=0.0, x0=case["phantom"] * 0.5)
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4


def test_batched_uneven_frames_equal_per_frame_solves(cuda):
    """Frames with different sample counts in one operator, solved with
    per-frame CG scalars (one launch per kernel for all frames), give the same
    images as one solve per frame."""
    N, mos, W, C = 32, 64, 5.5, 4
    spokes = [7, 13, 5, 11]
    trajs = [S.radial_golden_angle_2d(s, 64, profile_offset=17 * f) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    sq = np.concatenate([np.sqrt(S.ramp_dcw(t)) for t in trajs]).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    F = len(spokes)
    ph = np.stack([S.ellipse_phantom((N, N), 8, 30 + f) for f in range(F)], 0)
    # data per frame from the oracle operator
    d = np.zeros((C, offs[-1]), np.complex64)
    for f in range(F):
        P = O.OraclePlan((N, N), (mos, mos), W)
        P.preprocess(trajs[f][None])
        Ef = O.OracleSense(P, csm, sq[offs[f]:offs[f + 1]][None])
        d[:, offs[f]:offs[f + 1]] = Ef.mult_M(ph[f:f + 1]).reshape(C, -1)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(torch.from_numpy(csm).to(cuda))
    E.set_dcw(torch.from_numpy(sq).to(cuda))
    E.preprocess(torch.from_numpy(traj).to(cuda), frame_offsets=offs)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(8)
    cg.set_tc_tolerance(0.0)
    cg.set_frame_independent(True)
    cg.set_use_graph(True)
    xb = cg.solve(torch.from_numpy(d).to(cuda)).cpu().numpy()
    for f in range(F):
        P = O.OraclePlan((N, N), (mos, mos), W)
        P.preprocess(trajs[f][None])
        Ef = O.OracleSense(P, csm, sq[offs[f]:offs[f + 1]][None])
        xr = O.cg_solve(Ef, d[:, offs[f]:offs[f + 1]][:, None, :], iterations=8, tc_tolerance=0.0)
        assert rel_l2(xb[f], xr[0]) <= 1e-4, f


def test_grid_schedules_bit_identical(cuda):
    """The normal operator's gridding schedules -- one CTA per work item
    (schedule 1; here the warp-specialized kernel on the interleaved sample
    layout) and one persistent work-queue launch (schedule 2) -- give
    forward, E^H E and CG results equal bit for bit, on uneven frames whose
    dense radial centres are split over several work items, and match the
    oracle."""
    N, mos, W, C = 32, 64, 5.5, 12
    spokes = [64, 7, 13, 40, 5]
    trajs = [S.radial_golden_angle_2d(s, 64, profile_offset=11 * f) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    sq = np.concatenate([np.sqrt(S.ramp_dcw(t)) for t in trajs]).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    F = len(spokes)
    rng = np.random.default_rng(61)
    x = (rng.standard_normal((F, N, N)) + 1j * rng.standard_normal((F, N, N))).astype(np.complex64)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(torch.from_numpy(csm).to(cuda))
    E.set_dcw(torch.from_numpy(sq).to(cuda))
    E.preprocess(torch.from_numpy(traj).to(cuda), frame_offsets=offs)
    plan = E.get_plan()
    xt = torch.from_numpy(x).to(cuda)
    d = torch.empty((C, offs[-1]), dtype=torch.complex64, device=cuda)
    E.mult_M(xt, d)
    outs, sols, fwd = {}, {}, {}
    for sched in (1, 2, 0):
        plan.set_grid_schedule(sched)
        assert plan.get_grid_schedule() == sched
        y = torch.empty_like(d)
        E.mult_M(xt, y)
        fwd[sched] = y.cpu().numpy()
        o = torch.empty_like(xt)
        E.mult_MH_M(xt, o)
        outs[sched] = o.cpu().numpy()
        cg = gb.cuCgSolver()
        cg.set_encoding_operator(E)
        cg.set_max_iterations(5)
        cg.set_tc_tolerance(0.0)
        cg.set_frame_independent(True)
        cg.set_use_graph(True)
        sols[sched] = cg.solve(d).cpu().numpy()
    assert np.array_equal(fwd[1], fwd[2]) and np.array_equal(fwd[0], fwd[1])
    assert np.array_equal(outs[1], outs[2]) and np.array_equal(outs[0], outs[1])
    assert np.array_equal(sols[1], sols[2]) and np.array_equal(sols[0], sols[1])
    for f in (0, 3):
        P = O.OraclePlan((N, N), (mos, mos), W)
        P.preprocess(trajs[f][None])
        Ef = O.OracleSense(P, csm, sq[offs[f]:offs[f + 1]][None])
        assert rel_l2(outs[2][f], Ef.mult_MH_M(x[f:f + 1])[0]) <= PARITY_TOL, f
    assert plan.device_errors() == 0
    with pytest.raises(RuntimeError):
        plan.set_grid_schedule(3)


@pytest.mark.parametrize("frames,coils", [(1, 16), (3, 12), (2, 5)])
def test_row_fused_iteration_matches_cooperative_tail(cuda, frames, coils):
    """2D CG with the x passes fused into the pad and the crop (the default;
    beta from the expanded norm of r - alpha q, the update folded into the
    next pad) against the barrier-synchronised fused tail (beta from the dot
    of the updated r): same iterates and residual history to rounding, both
    at the oracle's FP64 CG; frame-independent solves with a preconditioner
    too."""
    case = sense_case(N=64, coils=coils, frames=frames, seed=41 + frames)
    E, orc = make_ops(case, cuda)
    d = orc.mult_M(case["phantom"]).astype(np.complex64)
    dt = torch.from_numpy(d.reshape(coils, -1)).to(cuda)
    P = torch.from_numpy(np.random.default_rng(7).uniform(0.5, 1.5, (frames, 64, 64)).astype(np.float32)).to(cuda)
    for precond in (None, P):
        sols, hists = {}, {}
        for fused in (True, False):
            cg = gb.cuCgSolver()
            cg.set_encoding_operator(E)
            cg.set_max_iterations(8)
            cg.set_tc_tolerance(0.0)
            cg.set_frame_independent(frames > 1)
            cg.set_use_graph(True)
            cg.set_row_fusion(fused)
            if precond is not None:
                cg.set_preconditioner(precond)
            sols[fused] = cg.solve(dt).cpu().numpy()
            hists[fused] = cg.residual_history[:8].cpu().numpy().copy()
        assert rel_l2(sols[True], sols[False]) <= 1e-5
        np.testing.assert_allclose(hists[True], hists[False], rtol=1e-4)
        if precond is None and frames == 1:   # (frame-independent solves: per-frame oracle elsewhere)
            xr = O.cg_solve(orc, d, iterations=8, tc_tolerance=0.0)
            assert rel_l2(sols[True], xr) <= 1e-4
    assert E.get_plan().device_errors() == 0


def test_image_operator_matches_oracle(cuda):
    """cuImageOperator::compute (imageOperator.h:27-45, cuImageOperator.h:35-62):
    same float formulas, same histogram offset."""
    rng = np.random.default_rng(21)
    z = (rng.standard_normal((2, 64, 64)) + 1j * rng.standard_normal((2, 64, 64))).astype(np.complex64)
    R = gb.cuImageOperator()
    R.compute(torch.from_numpy(z).to(cuda))
    ref, off = O.image_operator_compute(z)
    assert abs(R.offset_ - off) <= 1e-6 * off
    np.testing.assert_allclose(R.get().cpu().numpy(), ref, rtol=2e-6)
    z2 = np.full(100, 4.0, np.complex64)
    z2[37] = 1.0
    R.compute(torch.from_numpy(z2).to(cuda))
    ref2, off2 = O.image_operator_compute(z2)
    assert R.offset_ == off2
    assert np.array_equal(R.get().cpu().numpy(), ref2)
    R.compute(torch.from_numpy(z).to(cuda), offset_estimation=False)
    ref3, off3 = O.image_operator_compute(z, offset_estimation=False)
    assert R.offset_ == 0.0 and off3 == 0.0
    np.testing.assert_allclose(R.get().cpu().numpy(), ref3, rtol=2e-6)


def test_sense_precond_weights_matches_oracle(cuda):
    case = sense_case(coils=8, seed=5)
    E, orc = make_ops(case, cuda)
    w0 = gb.sense_precond_weights(E)
    np.testing.assert_allclose(w0.cpu().numpy(), O.sense_precond_weights(case["csm"]), rtol=2e-6)
    rng = np.random.default_rng(6)
    reg = rng.uniform(0.5, 3.0, (64, 64)).astype(np.float32)
    w1 = gb.sense_precond_weights(E, torch.from_numpy(reg).to(cuda), kappa=0.3)
    np.testing.assert_allclose(w1.cpu().numpy(), O.sense_precond_weights(case["csm"], reg, 0.3), rtol=2e-6)


@pytest.mark.parametrize("frames,use_graph", [(1, False), (1, True), (2, False)])
def test_cg_image_regularization_and_preconditioner(cuda, frames, use_graph):
    """The gpuCgSenseGadget solve (gpuCgSenseGadget.cpp:65-77,164-190): image
    regulariser of weight kappa from a regularisation image, preconditioner
    1/sqrt(sum |csm|^2 + kappa R), CG on (E^H E + kappa R^H R) x = E^H d."""
    case = sense_case(coils=8, seed=7, frames=frames)
    E, orc = make_ops(case, cuda)
    d_ref = orc.mult_M(case["phantom"])
    rng = np.random.default_rng(8)
    noise = 0.02 * np.sqrt(np.mean(np.abs(d_ref) ** 2)) * (rng.standard_normal(d_ref.shape) +
                                                          1j * rng.standard_normal(d_ref.shape)) / np.sqrt(2)
    d = (d_ref + noise).astype(np.complex64)
    d_t = torch.from_numpy(d.reshape(8, -1)).to(cuda)
    kappa = 0.05
    # regularisation image: the first frame's adjoint reconstruction (the
    # gadget takes it from the rhs buffer), one frame broadcast over frames
    reg_all = torch.empty((frames, 64, 64), dtype=torch.complex64, device=cuda)
    E.mult_MH(d_t, reg_all)
    reg = reg_all[0].contiguous()
    R = gb.cuImageOperator()
    R.compute(reg)
    R.set_weight(kappa)
    D = gb.cuCgPreconditioner()
    D.set_weights(gb.sense_precond_weights(E, R.get(), kappa))
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.add_regularization_operator(R)
    cg.set_preconditioner(D)
    cg.set_max_iterations(10)
    cg.set_tc_tolerance(0.0)
    cg.set_use_graph(use_graph)
    x = cg.solve(d_t)
    R_o, _ = O.image_operator_compute(reg.cpu().numpy())
    w_o = O.sense_precond_weights(case["csm"], R_o, kappa)
    xr = O.cg_solve(orc, d, iterations=10, tc_tolerance=0.0, precond_weights=w_o[None],
                    regularization=[(kappa, R_o[None])])
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4
    # the regulariser is active: the unregularised solution is measurably different
    xu = O.cg_solve(orc, d, iterations=10, tc_tolerance=0.0, precond_weights=w_o[None])
    assert rel_l2(xu, xr) > 1e-3
    if use_graph:
        assert torch.equal(x, cg.solve(d_t))
    assert E.get_plan().device_errors() == 0


def test_grid_barrier_timeout_flags_error_and_next_solve_recovers(cuda):
    """The fused CG tail's grid barrier is a bounded wait (2D plans take it
    with the row fusion off; 3D plans always).  With its limit set to one
    poll, blocks give up instead of waiting: the solve returns, the device
    error word reports bit 1, and nothing hangs.  Solves after it at the
    default limit (plain and graph-captured) start from cleared barrier
    counters and match the oracle again."""
    case = sense_case(coils=4, seed=31)
    E, orc = make_ops(case, cuda)
    d = orc.mult_M(case["phantom"]).astype(np.complex64)
    dt = torch.from_numpy(d.reshape(4, -1)).to(cuda)
    cg = gb.cuCgSolver()
    cg.set_row_fusion(False)
    cg.set_encoding_operator(E)
    cg.set_max_iterations(6)
    cg.set_tc_tolerance(0.0)
    assert E.get_plan().device_errors() == 0
    cg.set_barrier_spin_limit(1)
    cg.solve(dt)
    torch.cuda.synchronize()
    assert E.get_plan().device_errors() & 2
    cg.set_barrier_spin_limit(0)
    xr = O.cg_solve(orc, d, iterations=6, tc_tolerance=0.0)
    for use_graph in (False, True):
        cg.set_use_graph(use_graph)
        x = cg.solve(dt)
        assert rel_l2(x.cpu().numpy(), xr) <= 1e-4
    assert E.get_plan().device_errors() == 0
