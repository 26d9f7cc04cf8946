"""Density compensation estimate (estimate_dcw, toolboxes/mri/sdc/SDC.hpp:19-80
and toolboxes/mri/sdc/gpu/cuSDC.cu) over the C ABI: iterative
w <- w / C2NC(NC2C(w)) with the Jinc kernel on the GPU."""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream


def estimate_dcw(traj: torch.Tensor, matrix_size: Sequence[int], os_factor: float, num_iterations: int,
                 kernel_width: float = 5.5, initial_dcw: Optional[torch.Tensor] = None) -> torch.Tensor:
    """traj: float32 [M, D] (or [..., D]) in [-1/2, 1/2]; returns float32 [M]."""
    _check_tensor(traj, torch.float32, "traj")
    D = len(matrix_size)
    if traj.numel() % D:
        raise ValueError("trajectory size is not a multiple of D")
    M = traj.numel() // D
    if initial_dcw is not None:
        _check_tensor(initial_dcw, torch.float32, "initial_dcw")
        if initial_dcw.numel() != M:
            raise ValueError("initial_dcw must hold one weight per sample")
    out = torch.empty(M, dtype=torch.float32, device=traj.device)
    n = (ctypes.c_uint64 * D)(*[int(v) for v in matrix_size])
    check(lib.gb_sdc_estimate_dcw(D, n, ctypes.c_float(os_factor), int(num_iterations), ctypes.c_float(kernel_width),
                                  _ptr(traj), M, _ptr(initial_dcw), _ptr(out), _stream()))
    return out
