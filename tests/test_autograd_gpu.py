"""Differentiation through the torch.autograd.Function wrappers (GPU).

* image gradient of the forward NUFFT = the adjoint, checked against the
  oracle's BACKWARDS_NC2C (the reference's mult_MH path);
* trajectory gradient (analytic derivative of the Kaiser-Bessel rational
  approximation) against central finite differences with step 1e-4 in k
  units, on 64 random samples, relative error <= 1e-3.  Every output sample
  depends only on its own trajectory point, so one +h / -h pair of forward
  evaluations per dimension gives every sample's directional derivative.
  Samples whose footprint gains or loses a tap inside [k-h, k+h] are excluded:
  there the reference kernel jumps (its edge value is I0(0) * mos / W).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from gadgetron_b200 import synthetic as S
from tests.helpers import PARITY_TOL, rel_l2

pytestmark = pytest.mark.gpu

import gadgetron_b200 as gb  # noqa: E402
from gadgetron_b200.autograd import nufft_adjoint, nufft_forward  # noqa: E402

FD_STEP = 1e-4
FD_TOL = 1e-3


def _valid_fd_samples(traj, mos, W, h):
    """Samples whose tap range is constant for every k in [k-h, k+h]."""
    r = W / 2.0
    ok = np.ones(traj.shape[0], bool)
    for d in range(traj.shape[1]):
        for sgn in (-1.0, 1.0):
            sp_lo = (traj[:, d].astype(np.float64) - h) * mos[d] + mos[d] / 2.0
            sp_hi = (traj[:, d].astype(np.float64) + h) * mos[d] + mos[d] / 2.0
            a = np.ceil(sp_lo + sgn * r - 1e-3)
            b = np.ceil(sp_hi + sgn * r + 1e-3)
            ok &= (a == b)
            a = np.floor(sp_lo + sgn * r - 1e-3)
            b = np.floor(sp_hi + sgn * r + 1e-3)
            ok &= (a == b)
    return np.nonzero(ok)[0]


def _fd_check(case_traj, N, mos, W, nb, seed, forward=True):
    dev = torch.device("cuda:0")
    # keep k +- h inside [-1/2, 1/2] (the radial spokes start at -1/2 exactly)
    case_traj = (case_traj.astype(np.float64) * 0.999).astype(np.float32)
    D = len(N)
    rng = np.random.default_rng(seed)
    M = case_traj.shape[0]
    dcw = S.ramp_dcw(case_traj)
    dcw_t = torch.from_numpy(dcw).to(dev)
    plan = gb.NFFT.make_plan(N, mos, W)
    traj_t = torch.from_numpy(case_traj).to(dev).requires_grad_(True)
    plan.preprocess(traj_t.detach())
    shape = (nb, 1) + tuple(reversed(N))
    if forward:
        x = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)).to(dev)
        v = torch.from_numpy((rng.standard_normal((nb, M)) + 1j * rng.standard_normal((nb, M))).astype(np.complex64)).to(dev)
        y = nufft_forward(x, traj_t, plan, dcw_t)
        loss = (v.conj() * y).real.sum()
    else:
        yin = torch.from_numpy((rng.standard_normal((nb, M)) + 1j * rng.standard_normal((nb, M))).astype(np.complex64)).to(dev)
        v = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)).to(dev)
        xo = nufft_adjoint(yin, traj_t, plan, dcw_t)
        loss = (v.conj() * xo).real.sum()
    loss.backward()
    g_ad = traj_t.grad.detach().cpu().numpy().astype(np.float64)

    # Finite differences: all samples shifted together along one dimension.
    g_fd = np.zeros((M, D))
    for d in range(D):
        vals = []
        for sgn in (1.0, -1.0):
            tp = case_traj.copy()
            tp[:, d] = (tp[:, d].astype(np.float64) + sgn * FD_STEP).astype(np.float32)
            p2 = gb.NFFT.make_plan(N, mos, W)
            p2.preprocess(torch.from_numpy(tp).to(dev))
            if forward:
                out = torch.empty((nb, M), dtype=torch.complex64, device=dev)
                p2.compute(x, out, dcw_t, gb.NFFT_comp_mode.FORWARDS_C2NC)
                contrib = (v.conj() * out).real.double().sum(0)      # per sample
            else:
                out = torch.empty(shape, dtype=torch.complex64, device=dev)
                # per-sample contribution: run the adjoint of one-hot weights is
                # too costly; use linearity: L = sum_j Re(<v, A^H e_j y_j>)
                # = sum_j Re(conj(A v)_j y_j) with A the forward at tp.
                av = torch.empty((nb, M), dtype=torch.complex64, device=dev)
                p2.compute(v, av, dcw_t, gb.NFFT_comp_mode.FORWARDS_C2NC)
                contrib = (av.conj() * yin).real.double().sum(0)
            vals.append(contrib.cpu().numpy())
        # float32 coordinates: use the realised step
        dk = (case_traj[:, d].astype(np.float64) + FD_STEP).astype(np.float32).astype(np.float64) - \
             (case_traj[:, d].astype(np.float64) - FD_STEP).astype(np.float32).astype(np.float64)
        g_fd[:, d] = (vals[0] - vals[1]) / dk
    valid = _valid_fd_samples(case_traj, mos, W, FD_STEP)
    pick = rng.choice(valid, 64, replace=False)
    err = np.linalg.norm(g_ad[pick] - g_fd[pick]) / np.linalg.norm(g_fd[pick])
    return err, len(valid) / M


def test_image_gradient_is_reference_adjoint(cuda):
    N, mos, W = (64, 64), (128, 128), 5.5
    traj = S.radial_golden_angle_2d(32, 128)
    dcw = S.ramp_dcw(traj)
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(cuda))
    rng = np.random.default_rng(0)
    x = torch.from_numpy((rng.standard_normal((2, 1, 64, 64)) + 1j * rng.standard_normal((2, 1, 64, 64)))
                         .astype(np.complex64)).to(cuda).requires_grad_(True)
    v = (rng.standard_normal((2, traj.shape[0])) + 1j * rng.standard_normal((2, traj.shape[0]))).astype(np.complex64)
    y = nufft_forward(x, torch.from_numpy(traj).to(cuda), plan, torch.from_numpy(dcw).to(cuda))
    (torch.from_numpy(v).to(cuda).conj() * y).real.sum().backward()
    orc = O.OraclePlan(N, mos, W)
    orc.preprocess(traj[None])
    ref = orc.backwards_nc2c(v, dcw[None])
    assert rel_l2(x.grad.cpu().numpy(), ref) <= PARITY_TOL


def test_traj_grad_fd_2d(cuda):
    traj = S.radial_golden_angle_2d(48, 128)
    err, frac = _fd_check(traj, (64, 64), (128, 128), 5.5, nb=3, seed=1)
    assert frac > 0.5
    assert err <= FD_TOL, err


def test_traj_grad_fd_3d(cuda):
    traj = S.kooshball_golden_means_3d(400, 64)
    err, frac = _fd_check(traj, (32, 32, 32), (64, 64, 64), 4.0, nb=4, seed=2)
    assert frac > 0.5
    assert err <= FD_TOL, err


def test_traj_grad_fd_adjoint_2d(cuda):
    traj = S.radial_golden_angle_2d(32, 128)
    err, _ = _fd_check(traj, (64, 64), (128, 128), 5.5, nb=2, seed=3, forward=False)
    assert err <= FD_TOL, err


def test_samples_gradient_of_adjoint(cuda):
    N, mos, W = (32, 32), (64, 64), 4.0
    traj = S.radial_golden_angle_2d(16, 64)
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(cuda))
    rng = np.random.default_rng(4)
    y = torch.from_numpy((rng.standard_normal((2, traj.shape[0])) + 1j * rng.standard_normal((2, traj.shape[0])))
                         .astype(np.complex64)).to(cuda).requires_grad_(True)
    v = (rng.standard_normal((2, 1, 32, 32)) + 1j * rng.standard_normal((2, 1, 32, 32))).astype(np.complex64)
    x = nufft_adjoint(y, torch.from_numpy(traj).to(cuda), plan, None)
    (torch.from_numpy(v).to(cuda).conj() * x).real.sum().backward()
    orc = O.OraclePlan(N, mos, W)
    orc.preprocess(traj[None])
    assert rel_l2(y.grad.cpu().numpy(), orc.forward_c2nc(v).reshape(2, -1)) <= PARITY_TOL


@pytest.mark.parametrize("dims", [2, 3])
def test_traj_grad_kernel_matches_oracle(cuda, dims):
    """The trajectory-derivative kernel against the oracle's FP64 restatement
    (same taps, float kernel values, analytic derivative of the rational
    approximation), through the C ABI."""
    if dims == 2:
        N, mos, W = (64, 64), (128, 128), 5.5
        traj = S.radial_golden_angle_2d(40, 128)
        shape = (3, 1, 64, 64)
    else:
        N, mos, W = (32, 32, 32), (64, 64, 64), 4.0
        traj = S.kooshball_golden_means_3d(300, 64)
        shape = (3, 1, 32, 32, 32)
    M = traj.shape[0]
    dcw = S.ramp_dcw(traj)
    rng = np.random.default_rng(11)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    w = (rng.standard_normal((3, M)) + 1j * rng.standard_normal((3, M))).astype(np.complex64)
    plan = gb.NFFT.make_plan(N, mos, W)
    plan.preprocess(torch.from_numpy(traj).to(cuda))
    g = plan.traj_grad(torch.from_numpy(x).to(cuda), torch.from_numpy(w).to(cuda),
                       torch.from_numpy(dcw).to(cuda)).cpu().numpy()
    orc = O.OraclePlan(N, mos, W)
    orc.preprocess(traj[None])
    ref = orc.traj_grad_forward(x, w, dcw[None])
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) <= 1e-4
