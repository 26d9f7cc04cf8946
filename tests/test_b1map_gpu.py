"""GPU parity of the coil sensitivity estimate (estimate_b1_map,
toolboxes/mri/pmri/gpu/b1_map.cu:29-118) against the oracle."""
import numpy as np
import pytest
import torch

from gadgetron_b200 import synthetic as S
from oracle import oracle as O
from tests.helpers import PARITY_TOL, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402


def _coil_images(shape, C, seed):
    rng = np.random.default_rng(seed)
    csm = S.gaussian_bump_csm(shape, C)
    rho = 1.0 + rng.uniform(0, 1, shape)
    noise = 0.01 * (rng.standard_normal((C,) + shape) + 1j * rng.standard_normal((C,) + shape))
    return (csm * rho[None] + noise).astype(np.complex64)


@pytest.mark.parametrize("shape,C,target", [((64, 64), 8, -1), ((48, 80), 12, 6), ((96, 96), 16, -1),
                                            ((50, 30), 3, -1), ((40, 36), 24, -1), ((32, 32), 20, 18)])
def test_b1_map_2d(cuda, shape, C, target):
    imgs = _coil_images(shape, C, 3)
    est = gb.b1map.estimate_b1_map(torch.from_numpy(imgs).to(cuda), 2, target)
    ref = O.estimate_b1_map(imgs, 2, target)
    assert est.shape == ref.shape
    assert rel_l2(est.cpu().numpy(), ref) <= PARITY_TOL


def test_b1_map_3d(cuda):
    imgs = _coil_images((16, 24, 20), 4, 7)
    est = gb.b1map.estimate_b1_map(torch.from_numpy(imgs).to(cuda), 3)
    assert rel_l2(est.cpu().numpy(), O.estimate_b1_map(imgs, 3)) <= PARITY_TOL


def test_b1_map_1d(cuda):
    rng = np.random.default_rng(11)
    x = np.linspace(-0.5, 0.5, 300, endpoint=False)
    C = 5
    mu = np.linspace(-0.4, 0.4, C)
    csm = np.exp(-((x[None] - mu[:, None]) ** 2) / (2 * 0.2 ** 2)) * np.exp(1j * rng.uniform(-np.pi, np.pi, (C, 1)))
    imgs = (csm * (1.0 + rng.uniform(0, 1, x.shape))[None] +
            0.01 * (rng.standard_normal((C, 300)) + 1j * rng.standard_normal((C, 300)))).astype(np.complex64)
    est = gb.b1map.estimate_b1_map(torch.from_numpy(imgs).to(cuda), 1)
    assert rel_l2(est.cpu().numpy(), O.estimate_b1_map(imgs, 1)) <= PARITY_TOL


def test_b1_map_repeated_calls_reuse_scratch(cuda):
    """Calls of different sizes in turn (the scratch grows and is reused)
    give the same results as the first call of each size."""
    big = torch.from_numpy(_coil_images((96, 96), 16, 5)).to(cuda)
    small = torch.from_numpy(_coil_images((40, 72), 6, 6)).to(cuda)
    first_big = gb.b1map.estimate_b1_map(big, 2)
    first_small = gb.b1map.estimate_b1_map(small, 2)
    for _ in range(2):
        assert torch.equal(gb.b1map.estimate_b1_map(big, 2), first_big)
        assert torch.equal(gb.b1map.estimate_b1_map(small, 2), first_small)


def test_b1_map_feeds_sense(cuda):
    """The estimate drives a SENSE operator like any coil map (unit norm per
    pixel over the coils)."""
    imgs = _coil_images((64, 64), 8, 9)
    est = gb.b1map.estimate_b1_map(torch.from_numpy(imgs).to(cuda), 2)
    nrm = est.abs().pow(2).sum(0).sqrt()
    assert torch.allclose(nrm, torch.ones_like(nrm), atol=1e-5)
