"""GPU parity of the SENSE accumulation buffer (cuSenseBuffer,
toolboxes/mri/pmri/gpu/cuBuffer.cpp:7-166 and cuSenseBuffer.cpp:18-35)
against the oracle, frame by frame."""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O
from tests.helpers import PARITY_TOL, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402


@pytest.mark.parametrize("use_dcw", [False, True])
def test_sense_buffer_matches_oracle(cuda, use_dcw):
    N, mos, W, C = (64, 64), (128, 128), 5.5, 4
    buf = gb.cuSenseBuffer()
    buf.setup(N, mos, W, C, num_cycles=2, num_sub_cycles=3)
    orc = O.OracleSenseBuffer(N, mos, W, C, num_cycles=2, num_sub_cycles=3)
    csm = S.gaussian_bump_csm(N, C)
    buf.set_csm(torch.from_numpy(csm).to(cuda))
    assert abs(buf.get_normalization_factor() - 1.0 / 6.0) < 1e-7
    # nothing accumulated yet: ones
    assert torch.all(buf.get_accumulated_coil_images() == 1)
    rng = np.random.default_rng(11)
    completed = 0
    for f in range(8):
        t = S.radial_golden_angle_2d(16, 128, profile_offset=16 * f).astype(np.float32)
        y = (rng.standard_normal((C, t.shape[0])) + 1j * rng.standard_normal((C, t.shape[0]))).astype(np.complex64)
        dcw = S.ramp_dcw(t).astype(np.float32)
        if use_dcw:
            d_t = torch.from_numpy(dcw).to(cuda)
            buf.set_dcw(d_t)
            orc.dcw = dcw
        done = buf.add_frame_data(torch.from_numpy(y).to(cuda), torch.from_numpy(t).to(cuda))
        assert done == orc.add_frame_data(y, t)
        if done:
            completed += 1
            img = buf.get_accumulated_coil_images()
            ref = orc.get_accumulated_coil_images()
            assert rel_l2(img.cpu().numpy(), ref) <= PARITY_TOL
            comb = buf.get_combined_coil_image()
            assert rel_l2(comb.cpu().numpy(), orc.get_combined_coil_image(csm)) <= PARITY_TOL
    assert completed == 2
    buf.clear()
    assert torch.all(buf.get_accumulated_coil_images() == 1)


def test_sense_buffer_errors(cuda):
    buf = gb.cuSenseBuffer()
    with pytest.raises(gb.GadgetronB200Error):
        buf.get_normalization_factor()            # no setup
    buf.setup((32, 32), (64, 64), 5.5, 2, 1, 1)
    with pytest.raises(gb.GadgetronB200Error):
        buf.get_combined_coil_image()             # no csm
