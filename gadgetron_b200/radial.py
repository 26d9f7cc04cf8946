"""Radial trajectories and density compensation weights generated on the
device: the Python mirror of toolboxes/core/gpu/radial_utilities.h:16-39
(compute_radial_trajectory_{golden_ratio,fixed_angle,variable_angle}_2d,
compute_radial_dcw_{golden_ratio,fixed_angle}_2d) over the C ABI.

Trajectories are float32 tensors [frames, profiles * samples, 2]; the dcw a
float32 tensor [profiles * samples] (one frame).
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream

GR_SMALLEST = 0
GR_ORIGINAL = 1


def _device(device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def compute_radial_trajectory_golden_ratio_2d(samples_per_profile: int, profiles_per_frame: int, frames: int = 1,
                                              profile_offset: int = 0, mode: int = GR_ORIGINAL,
                                              device=None) -> torch.Tensor:
    out = torch.empty((frames, profiles_per_frame * samples_per_profile, 2), dtype=torch.float32,
                      device=_device(device))
    check(lib.gb_radial_trajectory_golden_ratio_2d(samples_per_profile, profiles_per_frame, frames, profile_offset,
                                                   int(mode), _ptr(out), _stream()))
    return out


def compute_radial_trajectory_fixed_angle_2d(samples_per_profile: int, profiles_per_frame: int, frames: int = 1,
                                             angular_offset: float = 0.0, device=None) -> torch.Tensor:
    out = torch.empty((frames, profiles_per_frame * samples_per_profile, 2), dtype=torch.float32,
                      device=_device(device))
    check(lib.gb_radial_trajectory_fixed_angle_2d(samples_per_profile, profiles_per_frame, frames,
                                                  ctypes.c_float(angular_offset), _ptr(out), _stream()))
    return out


def compute_radial_trajectory_variable_angle_2d(angles: torch.Tensor, samples_per_profile: int,
                                                profiles_per_frame: int, frames: int) -> torch.Tensor:
    _check_tensor(angles, torch.float32, "angles")
    if angles.numel() < frames:
        raise ValueError("one angle per frame is needed")
    out = torch.empty((frames, profiles_per_frame * samples_per_profile, 2), dtype=torch.float32,
                      device=angles.device)
    check(lib.gb_radial_trajectory_variable_angle_2d(_ptr(angles), samples_per_profile, profiles_per_frame, frames,
                                                     _ptr(out), _stream()))
    return out


def compute_radial_dcw_golden_ratio_2d(samples_per_profile: int, profiles: int, alpha: float,
                                       one_over_radial_oversampling_factor: float, profile_offset: int = 0,
                                       mode: int = GR_ORIGINAL, device=None) -> torch.Tensor:
    out = torch.empty(profiles * samples_per_profile, dtype=torch.float32, device=_device(device))
    check(lib.gb_radial_dcw_golden_ratio_2d(samples_per_profile, profiles, ctypes.c_float(alpha),
                                            ctypes.c_float(one_over_radial_oversampling_factor), profile_offset,
                                            int(mode), _ptr(out), _stream()))
    return out


def compute_radial_dcw_fixed_angle_2d(samples_per_profile: int, profiles: int, alpha: float,
                                      one_over_radial_oversampling_factor: float, device=None) -> torch.Tensor:
    out = torch.empty(profiles * samples_per_profile, dtype=torch.float32, device=_device(device))
    check(lib.gb_radial_dcw_fixed_angle_2d(samples_per_profile, profiles, ctypes.c_float(alpha),
                                           ctypes.c_float(one_over_radial_oversampling_factor), _ptr(out),
                                           _stream()))
    return out
