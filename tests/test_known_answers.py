"""Known-answer checks taken from the reference's own tests for this path.

* test/cuNFFT_test.cpp:23-117 sets up 2500 x 1100 samples, all at
  k = (0.1, 0.1), unit data and unit density weights, 8 coils, a 256x256
  image oversampled to 544x544 (2.1 x 256 rounded up to the warp size), W = 3,
  and runs BACKWARDS_NC2C (it checks only that STANDARD finishes in < 20 s and
  ATOMIC in < 2 s).  Its answer is analytic: every coil image is
  M / sqrt(544^2) * exp(+2 pi i 0.1 ((x - 128) + (y - 128))), up to the
  kernel's approximation error at W = 3.
* test/cuNDFFT_test.cpp:35-47: the centred unitary FFT preserves the L2 norm
  of a 128^3 array to 1e-3 (forward and inverse).
"""
import time

import numpy as np
import pytest

from oracle import oracle as O

N, MOS, W = 256, 544, 3.0
RO, INT, CHA = 2500, 1100, 8
M = RO * INT
APPROX_TOL = 1e-2      # Kaiser-Bessel W = 3 approximation error (oracle: 5.3e-3)


def analytic_image():
    n = np.arange(N)
    ph = np.exp(2j * np.pi * 0.1 * ((n[None, :] - N // 2) + (n[:, None] - N // 2)))
    return (M / np.sqrt(MOS * MOS)) * ph


def test_oracle_constant_trajectory_known_answer():
    traj = np.full((1, M, 2), 0.1, np.float32)
    P = O.OraclePlan((N, N), (MOS, MOS), W)
    P.preprocess(traj)
    y = np.ones((2, 1, M), np.complex64)      # two of the eight coils (identical)
    x = P.backwards_nc2c(y, np.ones((1, M), np.float32))
    ana = analytic_image()
    assert O.rel_l2(x[0, 0], ana) < APPROX_TOL
    assert O.rel_l2(x[1, 0], ana) < APPROX_TOL


def test_oracle_centred_fft_preserves_norm():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((128, 128, 128)) + 1j * rng.standard_normal((128, 128, 128))
    n0 = np.linalg.norm(a)
    assert abs(np.linalg.norm(O.centred_fft(a, 3, True)) - n0) < 1e-3 * n0
    assert abs(np.linalg.norm(O.centred_fft(a, 3, False)) - n0) < 1e-3 * n0


@pytest.mark.gpu
@pytest.mark.parametrize("compensated", [False, True])
def test_gpu_constant_trajectory_known_answer(cuda, compensated):
    import torch
    import gadgetron_b200 as gb
    flags = gb.FLAG_COMPENSATED if compensated else 0
    traj = torch.full((M, 2), 0.1, dtype=torch.float32, device=cuda)
    data = torch.ones((CHA, M), dtype=torch.complex64, device=cuda)
    dcw = torch.ones(M, dtype=torch.float32, device=cuda)
    out = torch.empty((CHA, 1, N, N), dtype=torch.complex64, device=cuda)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan = gb.NFFT.make_plan((N, N), (MOS, MOS), W, flags=flags)
    plan.preprocess(traj, gb.NFFT_prep_mode.NC2C)
    plan.compute(data, out, dcw, gb.NFFT_comp_mode.BACKWARDS_NC2C)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert elapsed < 2.0        # the reference's bound for its fastest (ATOMIC) mode
    x = out.cpu().numpy()
    ana = analytic_image()
    for c in range(CHA):
        assert O.rel_l2(x[c, 0], ana) < APPROX_TOL
    # against the oracle (FP64 sums): 2.75M samples pile onto the same cells,
    # so plain FP32 sums drift; compensated sums stay at the parity bound
    P = O.OraclePlan((N, N), (MOS, MOS), W)
    P.preprocess(np.full((1, M, 2), 0.1, np.float32))
    ref = P.backwards_nc2c(np.ones((1, 1, M), np.complex64), np.ones((1, M), np.float32))[0, 0]
    err = O.rel_l2(x[0, 0], ref)
    assert err < (1e-5 if compensated else 1e-3), err


@pytest.mark.gpu
def test_gpu_fft_preserves_norm(cuda):
    import torch
    import gadgetron_b200 as gb
    plan = gb.NFFT.make_plan((128, 128, 128), (128, 128, 128), 4.0)
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((128, 128, 128)) + 1j * rng.standard_normal((128, 128, 128))).astype(np.complex64)
    n0 = np.linalg.norm(a)
    for mode in (gb.NFFT_fft_mode.FORWARDS, gb.NFFT_fft_mode.BACKWARDS):
        t = torch.from_numpy(a).to(cuda)
        plan.fft(t, mode)
        assert abs(np.linalg.norm(t.cpu().numpy()) - n0) < 1e-3 * n0
