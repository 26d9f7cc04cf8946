"""torch.autograd.Function wrappers of the NUFFT over the same C ABI.

This is the Python-layer entry to the path (the role Gadgetron's Python
gadget layer plays for the reference; the reference itself has no GPU
Python binding).  Gradients follow PyTorch's convention for complex tensors
(grad = dL/d(re) + i dL/d(im) for a real loss L):

* ``nufft_forward(image, traj, plan, dcw)`` computes y = dcw * NUFFT_k(image)
  (NFFT_comp_mode::FORWARDS_C2NC).  Backward: grad_image = A^H grad_y (the
  adjoint, BACKWARDS_NC2C with the same dcw) and
  grad_traj[j, d] = sum_b Re(conj(grad_y[b, j]) * d y[b, j] / d k[j, d]) from
  the hand-written trajectory-derivative kernel (analytic derivative of the
  Kaiser-Bessel rational approximation the reference uses).
* ``nufft_adjoint(samples, traj, plan, dcw)`` computes x = A^H samples
  (BACKWARDS_NC2C).  Backward: grad_samples = A grad_x and
  grad_traj[j, d] = sum_b Re(conj(dcw_j samples[b, j]) * sum_g d phi(s_j - g)/d k_d * K[b, g])
  where K is the forward grid of grad_x (same kernel).

The trajectory gradient is exact away from the points where a tap enters or
leaves the kernel support (the reference kernel is non-zero at its edge,
I0(0) * mos / W, so the operator jumps there).

The plan must have been preprocessed with ``traj`` (the trajectory values are
read from the plan; ``traj`` is the autograd handle).
"""
from __future__ import annotations

from typing import Optional

import torch

from .nfft import NFFT_comp_mode, cuNFFT_plan


class _NufftForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, traj, plan: cuNFFT_plan, dcw):
        nb = image.numel() // (plan.num_frames * _prod(plan.matrix_size))
        y = torch.empty((nb, plan.num_samples), dtype=torch.complex64, device=image.device)
        plan.compute(image.contiguous(), y, dcw, NFFT_comp_mode.FORWARDS_C2NC)
        ctx.plan = plan
        ctx.save_for_backward(image, dcw if dcw is not None else torch.empty(0))
        ctx.has_dcw = dcw is not None
        return y

    @staticmethod
    def backward(ctx, grad_y):
        image, dcw = ctx.saved_tensors
        dcw = dcw if ctx.has_dcw else None
        plan = ctx.plan
        grad_y = grad_y.resolve_conj().resolve_neg().contiguous()
        g_img = g_traj = None
        if ctx.needs_input_grad[0]:
            g_img = torch.empty_like(image)
            plan.compute(grad_y, g_img, dcw, NFFT_comp_mode.BACKWARDS_NC2C)
        if ctx.needs_input_grad[1]:
            g_traj = plan.traj_grad(image.contiguous(), torch.conj_physical(grad_y).contiguous(), dcw)
        return g_img, g_traj, None, None


class _NufftAdjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, samples, traj, plan: cuNFFT_plan, dcw):
        nb = samples.numel() // plan.num_samples
        shape = (nb, plan.num_frames) + tuple(reversed(plan.matrix_size))
        x = torch.empty(shape, dtype=torch.complex64, device=samples.device)
        plan.compute(samples.contiguous(), x, dcw, NFFT_comp_mode.BACKWARDS_NC2C)
        ctx.plan = plan
        ctx.save_for_backward(samples, dcw if dcw is not None else torch.empty(0))
        ctx.has_dcw = dcw is not None
        return x

    @staticmethod
    def backward(ctx, grad_x):
        samples, dcw = ctx.saved_tensors
        dcw = dcw if ctx.has_dcw else None
        plan = ctx.plan
        grad_x = grad_x.resolve_conj().resolve_neg().contiguous()
        g_s = g_traj = None
        if ctx.needs_input_grad[0]:
            g_s = torch.empty_like(samples)
            plan.compute(grad_x, g_s, dcw, NFFT_comp_mode.FORWARDS_C2NC)
        if ctx.needs_input_grad[1]:
            g_traj = plan.traj_grad(grad_x, torch.conj_physical(samples).contiguous(), dcw)
        return g_s, g_traj, None, None


def _prod(v):
    p = 1
    for a in v:
        p *= int(a)
    return p


def nufft_forward(image: torch.Tensor, traj: torch.Tensor, plan: cuNFFT_plan,
                  dcw: Optional[torch.Tensor] = None) -> torch.Tensor:
    return _NufftForward.apply(image, traj, plan, dcw)


def nufft_adjoint(samples: torch.Tensor, traj: torch.Tensor, plan: cuNFFT_plan,
                  dcw: Optional[torch.Tensor] = None) -> torch.Tensor:
    return _NufftAdjoint.apply(samples, traj, plan, dcw)
