"""Python mirrors of the regularisation and preconditioning pieces that
``gpuCgSenseGadget`` puts around the CG-SENSE solve
(gadgets/pmri/gpuCgSenseGadget.cpp:65-77,164-176):

* ``cuImageOperator`` -- toolboxes/operators/gpu/cuImageOperator.h and
  toolboxes/operators/imageOperator.h: a diagonal regulariser
  R = diag(image), image = 1 / (|reg * n / asum(reg)| + offset), with
  R^H R = diag(image^2);
* ``cuCgPreconditioner`` -- toolboxes/solvers/cgPreconditioner.h:24-39: real
  diagonal weights applied twice per CG iteration;
* ``sense_precond_weights`` -- the gadget's weights
  1 / sqrt(sum_c |csm_c|^2 + kappa * image).

All arithmetic runs in libgadgetron_b200.so through the C ABI.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream


class cuImageOperator:
    def __init__(self):
        self.image_: Optional[torch.Tensor] = None
        self.offset_ = 0.0
        self.weight = 1.0

    # generalOperator::set_weight / get_weight
    def set_weight(self, w: float):
        self.weight = float(w)

    def get_weight(self) -> float:
        return self.weight

    # imageOperator::compute (imageOperator.h:27-45)
    def compute(self, image: torch.Tensor, offset_estimation: bool = True):
        _check_tensor(image, torch.complex64, "image")
        out = torch.empty(image.shape, dtype=torch.float32, device=image.device)
        off = ctypes.c_float()
        check(lib.gb_image_operator_compute(_ptr(image), image.numel(), int(bool(offset_estimation)), _ptr(out),
                                            ctypes.byref(off), _stream()))
        self.image_ = out
        self.offset_ = float(off.value)

    # imageOperator::get (imageOperator.h:24-25)
    def get(self) -> torch.Tensor:
        if self.image_ is None:
            raise RuntimeError("imageOperator: compute() has not been called")
        return self.image_

    # mult_M / mult_MH / mult_MH_M (imageOperator.h:48-84), elementwise
    def mult_M(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, accumulate: bool = False):
        y = x * self.get()
        return y if out is None else (out.add_(y) if accumulate else out.copy_(y))

    def mult_MH(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, accumulate: bool = False):
        return self.mult_M(x, out, accumulate)

    def mult_MH_M(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, accumulate: bool = False):
        y = (x * self.get()) * self.get()
        return y if out is None else (out.add_(y) if accumulate else out.copy_(y))


class cuCgPreconditioner:
    """cgPreconditioner::set_weights: real diagonal weights (a complex tensor
    contributes its real part, as real_to_complex weights do)."""

    def __init__(self):
        self.weights: Optional[torch.Tensor] = None

    def set_weights(self, w: torch.Tensor):
        if w.is_complex():
            w = w.real
        self.weights = w.to(torch.float32).contiguous()

    def get_weights(self) -> Optional[torch.Tensor]:
        return self.weights


def sense_precond_weights(E, reg_image: Optional[torch.Tensor] = None, kappa: float = 0.0) -> torch.Tensor:
    """1 / sqrt(sum_c |csm_c|^2 + kappa * reg_image) over the operator's pixels
    (gpuCgSenseGadget.cpp:167-176); reg_image: the regulariser image of one
    frame (R.get()) or None."""
    n = 1
    for v in E.matrix_size:
        n *= int(v)
    if reg_image is not None:
        _check_tensor(reg_image, torch.float32, "reg_image")
        if reg_image.numel() != n:
            raise ValueError("regularisation image must hold one frame of the operator's pixels")
    dev = E.csm.device if getattr(E, "csm", None) is not None else torch.device("cuda:0")
    w = torch.empty(tuple(reversed(E.matrix_size)), dtype=torch.float32, device=dev)
    check(lib.gb_sense_precond_weights(E._h, _ptr(reg_image), ctypes.c_float(kappa), _ptr(w), _stream()))
    return w
