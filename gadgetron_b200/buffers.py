"""Python mirror of cuSenseBuffer<float, D> (toolboxes/mri/pmri/gpu/cuSenseBuffer.h,
cuBuffer.h:13-57) over the C ABI: the cyclic k-space accumulation buffer that
real-time SENSE pipelines use to form coil images (for coil sensitivity
estimation and the regularisation image) from a sliding window of frames."""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from ._lib import check, lib
from .nfft import _check_tensor, _ptr, _stream


class cuSenseBuffer:
    def __init__(self):
        h = ctypes.c_void_p()
        check(lib.gb_sense_buffer_create(ctypes.byref(h)))
        self._h = h
        self.matrix_size = None
        self.num_coils = 0
        self.dcw = None
        self.csm = None
        self._device = None

    def __del__(self):
        if getattr(self, "_h", None) is not None and lib is not None:
            lib.gb_sense_buffer_destroy(self._h)
            self._h = None

    # cuBuffer::setup (cuBuffer.cpp:29-61)
    def setup(self, matrix_size: Sequence[int], matrix_size_os: Sequence[int], W: float, num_coils: int,
              num_cycles: int, num_sub_cycles: int, device=None):
        D = len(matrix_size)
        n = (ctypes.c_uint64 * D)(*[int(v) for v in matrix_size])
        m = (ctypes.c_uint64 * D)(*[int(v) for v in matrix_size_os])
        self._device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(self._device):
            check(lib.gb_sense_buffer_setup(self._h, D, n, m, ctypes.c_float(W), int(num_coils), int(num_cycles),
                                            int(num_sub_cycles), _stream()))
        self.matrix_size = tuple(int(v) for v in matrix_size)
        self.num_coils = int(num_coils)

    def clear(self):
        check(lib.gb_sense_buffer_clear(self._h, _stream()))

    def set_dcw(self, dcw: Optional[torch.Tensor]):
        if dcw is not None:
            _check_tensor(dcw, torch.float32, "dcw")
        self.dcw = dcw
        check(lib.gb_sense_buffer_set_dcw(self._h, _ptr(dcw)))

    def set_csm(self, csm: torch.Tensor):
        _check_tensor(csm, torch.complex64, "csm")
        self.csm = csm
        check(lib.gb_sense_buffer_set_csm(self._h, _ptr(csm)))

    # cuBuffer::add_frame_data (cuBuffer.cpp:63-134): True when a cycle completed
    def add_frame_data(self, samples: torch.Tensor, trajectory: torch.Tensor) -> bool:
        _check_tensor(samples, torch.complex64, "samples")
        _check_tensor(trajectory, torch.float32, "trajectory")
        D = len(self.matrix_size)
        M = trajectory.numel() // D
        if samples.numel() != M * self.num_coils:
            raise RuntimeError("cuBuffer::add_frame_data: unexpected number of coils according to setup")
        if self.dcw is not None and self.dcw.numel() != M:
            raise RuntimeError("cuBuffer::add_frame_data: dcw does not match the frame's samples")
        done = ctypes.c_int()
        check(lib.gb_sense_buffer_add_frame_data(self._h, _ptr(samples), _ptr(trajectory), M, ctypes.byref(done),
                                                 _stream()))
        return bool(done.value)

    # cuBuffer::get_accumulated_coil_images (cuBuffer.cpp:136-166)
    def get_accumulated_coil_images(self) -> torch.Tensor:
        out = torch.empty((self.num_coils,) + tuple(reversed(self.matrix_size)), dtype=torch.complex64,
                          device=self._device)
        check(lib.gb_sense_buffer_get_accumulated_coil_images(self._h, _ptr(out), _stream()))
        return out

    # cuSenseBuffer::get_combined_coil_image (cuSenseBuffer.cpp:18-35)
    def get_combined_coil_image(self) -> torch.Tensor:
        out = torch.empty(tuple(reversed(self.matrix_size)), dtype=torch.complex64, device=self._device)
        check(lib.gb_sense_buffer_get_combined_coil_image(self._h, _ptr(out), _stream()))
        return out

    def get_normalization_factor(self) -> float:
        f = ctypes.c_float()
        check(lib.gb_sense_buffer_get_normalization_factor(self._h, ctypes.byref(f)))
        return float(f.value)
