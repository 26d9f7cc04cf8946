"""GPU parity of the density compensation estimate (estimate_dcw,
toolboxes/mri/sdc/SDC.hpp:19-80 with the Jinc kernel) against the oracle.
The device grids with float atomics and sums in float; the oracle sums in
FP64, hence relative-L2 tolerances."""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402


@pytest.mark.parametrize("N,os_factor,iters,kw", [((64, 64), 2.0, 10, 5.5), ((48, 80), 1.5, 5, 4.0),
                                                  ((64, 64), 3.0, 20, 5.5)])
def test_sdc_2d_matches_oracle(cuda, N, os_factor, iters, kw):
    traj = S.radial_golden_angle_2d(32, 128).astype(np.float32)
    w = gb.sdc.estimate_dcw(torch.from_numpy(traj).to(cuda), N, os_factor, iters, kw)
    ref = O.estimate_dcw(traj, N, os_factor, iters, kw)
    assert O.rel_l2(w.cpu().numpy(), ref) <= 1e-5


def test_sdc_3d_and_initial_weights(cuda):
    traj = S.kooshball_golden_means_3d(200, 32).astype(np.float32)
    init = S.ramp_dcw(traj).astype(np.float32)
    w = gb.sdc.estimate_dcw(torch.from_numpy(traj).to(cuda), (32, 32, 32), 2.0, 4, 4.0,
                            initial_dcw=torch.from_numpy(init).to(cuda))
    ref = O.estimate_dcw(traj, (32, 32, 32), 2.0, 4, 4.0, initial_dcw=init)
    assert O.rel_l2(w.cpu().numpy(), ref) <= 1e-5


def test_sdc_rejects_out_of_range(cuda):
    traj = torch.tensor([[0.2, 0.7]], dtype=torch.float32, device=cuda)
    with pytest.raises(gb.TrajectoryRangeError):
        gb.sdc.estimate_dcw(traj, (32, 32), 2.0, 2)


def test_sdc_repeated_calls_and_call_after_rejection(cuda):
    """Calls of changing grid sizes in turn, and a call after a rejected
    trajectory, reuse the kept scratch and still match the oracle."""
    small = S.radial_golden_angle_2d(16, 64).astype(np.float32)
    big = S.radial_golden_angle_2d(32, 128).astype(np.float32)
    cases = [(big, (96, 96)), (small, (32, 32)), (big, (96, 96))]
    for traj, N in cases:
        w = gb.sdc.estimate_dcw(torch.from_numpy(traj).to(cuda), N, 2.0, 5, 5.5)
        assert O.rel_l2(w.cpu().numpy(), O.estimate_dcw(traj, N, 2.0, 5, 5.5)) <= 1e-5
    bad = torch.tensor([[0.2, 0.7]], dtype=torch.float32, device=cuda)
    with pytest.raises(gb.TrajectoryRangeError):
        gb.sdc.estimate_dcw(bad, (32, 32), 2.0, 2)
    w = gb.sdc.estimate_dcw(torch.from_numpy(small).to(cuda), (32, 32), 2.0, 5, 5.5)
    assert O.rel_l2(w.cpu().numpy(), O.estimate_dcw(small, (32, 32), 2.0, 5, 5.5)) <= 1e-5
