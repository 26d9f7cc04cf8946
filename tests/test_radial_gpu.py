"""GPU parity of the device-side radial trajectory and density compensation
generators (toolboxes/core/gpu/radial_utilities.cu restated in
oracle/oracle.py).  Float32 arithmetic on both sides; the device uses CUDA's
sincosf, the oracle numpy's float32 sin/cos, hence the tolerances."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402
from gadgetron_b200 import radial as R  # noqa: E402


def _close(a, ref):
    """Positions in [-0.5, 0.5): within 1e-6 relative L2 overall and 1e-5 per
    coordinate (sin/cos of angles up to a few hundred radians differ in the
    last float bit between CUDA and numpy)."""
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    assert np.linalg.norm(a - ref) <= 1e-6 * np.linalg.norm(ref)
    assert np.abs(a - ref).max() <= 1e-5


@pytest.mark.parametrize("mode", [R.GR_SMALLEST, R.GR_ORIGINAL])
def test_golden_ratio_trajectory(cuda, mode):
    t = R.compute_radial_trajectory_golden_ratio_2d(256, 48, frames=3, profile_offset=5, mode=mode)
    ref = O.radial_trajectory_golden_ratio_2d(256, 48, 3, 5, mode)
    _close(t.cpu().numpy(), ref)


def test_fixed_and_variable_angle_trajectories(cuda):
    t = R.compute_radial_trajectory_fixed_angle_2d(128, 24, frames=4, angular_offset=0.3)
    _close(t.cpu().numpy(), O.radial_trajectory_fixed_angle_2d(128, 24, 4, 0.3))
    ang = torch.tensor([0.1, 1.2, -2.0], dtype=torch.float32, device=cuda)
    v = R.compute_radial_trajectory_variable_angle_2d(ang, 64, 8, 3)
    _close(v.cpu().numpy(), O.radial_trajectory_variable_angle_2d(ang.cpu().numpy(), 64, 8, 3))


@pytest.mark.parametrize("golden,mode,offset", [(True, R.GR_ORIGINAL, 0), (True, R.GR_SMALLEST, 7),
                                                (False, R.GR_ORIGINAL, 0)])
def test_radial_dcw(cuda, golden, mode, offset):
    S, P, alpha, ovs = 256, 40, 2.0, 0.5
    if golden:
        w = R.compute_radial_dcw_golden_ratio_2d(S, P, alpha, ovs, offset, mode)
    else:
        w = R.compute_radial_dcw_fixed_angle_2d(S, P, alpha, ovs)
    ref = O.radial_dcw_2d(S, P, alpha, ovs, offset, golden, mode)
    np.testing.assert_allclose(w.cpu().numpy(), ref, rtol=1e-4, atol=1e-7)


def test_radial_errors(cuda):
    with pytest.raises(gb.GadgetronB200Error):
        R.compute_radial_trajectory_golden_ratio_2d(100, 8)        # not a multiple of the warp size
    with pytest.raises(gb.GadgetronB200Error):
        R.compute_radial_dcw_fixed_angle_2d(128, 3, 1.0, 1.0)      # fewer than four profiles


def test_generated_inputs_drive_the_reconstruction(cuda):
    """The gadget path: device trajectory + device dcw into the SENSE operator,
    against the oracle fed the same arrays."""
    S, P, N = 256, 64, 64
    traj = R.compute_radial_trajectory_golden_ratio_2d(S, P)
    dcw = R.compute_radial_dcw_golden_ratio_2d(S, P, 2.0, 0.5)
    plan = gb.NFFT.make_plan((N, N), (2 * N, 2 * N), 5.5)
    plan.preprocess(traj.reshape(-1, 2).contiguous(), gb.NFFT_prep_mode.ALL)
    rng = np.random.default_rng(3)
    y = (rng.standard_normal((1, S * P)) + 1j * rng.standard_normal((1, S * P))).astype(np.complex64)
    out = torch.empty((1, 1, N, N), dtype=torch.complex64, device=cuda)
    plan.compute(torch.from_numpy(y).to(cuda), out, dcw, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    orc = O.OraclePlan((N, N), (2 * N, 2 * N), 5.5)
    orc.preprocess(traj.cpu().numpy().reshape(1, -1, 2))
    ref = orc.backwards_nc2c(y, dcw.cpu().numpy().reshape(1, -1))
    from tests.helpers import PARITY_TOL, rel_l2
    assert rel_l2(out.cpu().numpy(), ref) <= PARITY_TOL
