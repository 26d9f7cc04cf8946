"""Coil sensitivity estimation (estimate_b1_map<float, D>,
toolboxes/mri/pmri/gpu/b1_map.h:14-20) over the C ABI."""
from __future__ import annotations

import ctypes

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream


def estimate_b1_map(coil_images: torch.Tensor, D: int, target_coils: int = -1) -> torch.Tensor:
    """coil_images: complex64 [coils, *image] (x last, D image dimensions);
    returns complex64 [target, *image]."""
    _check_tensor(coil_images, torch.complex64, "coil_images")
    if coil_images.dim() != D + 1:
        raise RuntimeError("estimate_b1_map:: dimensionality mismatch.")
    nc = coil_images.shape[0]
    nt = nc if (target_coils <= 0 or target_coils > nc) else target_coils
    image = tuple(coil_images.shape[1:])
    dims = (ctypes.c_uint64 * D)(*[int(v) for v in reversed(image)])
    out = torch.empty((nt,) + image, dtype=torch.complex64, device=coil_images.device)
    check(lib.gb_estimate_b1_map(D, dims, nc, int(target_coils), _ptr(coil_images), _ptr(out), _stream()))
    return out
