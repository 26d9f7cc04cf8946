"""The radial SENSE pipeline around the solve, end to end on the GPU, against
the same chain on the oracle: golden-ratio trajectories and Voronoi weights
generated on the device (radial_utilities.cu), frames accumulated in the
SENSE buffer (cuBuffer.cpp), coil maps estimated from the accumulated coil
images (b1_map.cu), the regularisation image from the combined image
(imageOperator.h), the gadget's preconditioner, and the regularised CG-SENSE
solve of the last frame (gpuCgSenseGadget.cpp:65-77,164-190)."""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402
from gadgetron_b200 import radial as R  # noqa: E402


def test_radial_sense_chain(cuda):
    N, mos, W, C, P, Sp, frames = (64, 64), (128, 128), 5.5, 6, 16, 128, 4
    csm_true = S.gaussian_bump_csm(N, C)
    ph = S.ellipse_phantom(N, 10, 21)
    # device-generated trajectories (one golden-ratio frame after another) and weights
    dcw = R.compute_radial_dcw_golden_ratio_2d(Sp, P, 2.0, 0.5)
    dcw_np = dcw.cpu().numpy()
    buf = gb.cuSenseBuffer()
    buf.setup(N, mos, W, C, num_cycles=2, num_sub_cycles=2)
    buf.set_dcw(dcw)
    orc_buf = O.OracleSenseBuffer(N, mos, W, C, num_cycles=2, num_sub_cycles=2)
    orc_buf.dcw = dcw_np
    rng = np.random.default_rng(5)
    trajs, datas = [], []
    for f in range(frames):
        t = R.compute_radial_trajectory_golden_ratio_2d(Sp, P, 1, profile_offset=f * P)[0].contiguous()
        t_np = t.cpu().numpy()
        plan = O.OraclePlan(N, mos, W)
        plan.preprocess(t_np.reshape(1, -1, 2))
        y = plan.forward_c2nc((csm_true * ph[None])[:, None]).reshape(C, -1)
        y = (y + 0.001 * np.abs(y).max() * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)))
        y = y.astype(np.complex64)
        buf.add_frame_data(torch.from_numpy(y).to(cuda), t)
        orc_buf.add_frame_data(y, t_np)
        trajs.append(t)
        datas.append(y)
    acc = buf.get_accumulated_coil_images()
    acc_o = orc_buf.get_accumulated_coil_images()
    assert rel_l2(acc.cpu().numpy(), acc_o) <= 1e-5
    csm = gb.b1map.estimate_b1_map(acc, 2)
    csm_o = O.estimate_b1_map(acc_o, 2)
    assert rel_l2(csm.cpu().numpy(), csm_o) <= 1e-5
    buf.set_csm(csm)
    reg = buf.get_combined_coil_image()
    reg_o = np.sum(np.conj(csm_o) * acc_o, axis=0)
    assert rel_l2(reg.cpu().numpy(), reg_o) <= 1e-5
    kappa = 0.05
    Rop = gb.cuImageOperator()
    Rop.compute(reg[None].contiguous())
    Rop.set_weight(kappa)
    R_o, _ = O.image_operator_compute(reg_o.astype(np.complex64)[None])
    # regularised solve of the last frame with sqrt(dcw) weighting, as the gadget does
    sq = torch.sqrt(dcw).contiguous()
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup(N, mos, W)
    E.set_csm(csm)
    E.set_dcw(sq)
    E.preprocess(trajs[-1])
    D = gb.cuCgPreconditioner()
    D.set_weights(gb.sense_precond_weights(E, Rop.get()[0].contiguous(), kappa))
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.add_regularization_operator(Rop)
    cg.set_preconditioner(D)
    cg.set_max_iterations(8)
    cg.set_tc_tolerance(0.0)
    d = (torch.from_numpy(datas[-1]).to(cuda) * sq[None]).contiguous()
    x = cg.solve(d)
    plan = O.OraclePlan(N, mos, W)
    plan.preprocess(trajs[-1].cpu().numpy().reshape(1, -1, 2))
    orc = O.OracleSense(plan, csm_o, sq.cpu().numpy()[None])
    w_o = O.sense_precond_weights(csm_o, R_o[0], kappa)
    xr = O.cg_solve(orc, d.cpu().numpy()[:, None, :], iterations=8, tc_tolerance=0.0, precond_weights=w_o[None],
                    regularization=[(kappa, R_o)])
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4
    assert E.get_plan().device_errors() == 0
