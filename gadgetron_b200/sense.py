"""Python mirror of ``cuNonCartesianSenseOperator<float,D>``
(toolboxes/mri/pmri/gpu/cuNonCartesianSenseOperator.h:12-41) over the C ABI.

Domain: images (frames, N_{D-1}, ..., N_0) complex64; codomain: samples
(coils, M_total) complex64; csm (coils, N_{D-1}, ..., N_0).  As in the
reference gadget, the density compensation passed to ``set_dcw`` is sqrt(w)
(gadgets/pmri/gpuCgSenseGadget.cpp:129).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from ._lib import check, lib
from .nfft import ConvolutionType, _check_tensor, _ptr, _stream, _u64, cuNFFT_plan


class cuNonCartesianSenseOperator:
    def __init__(self, D: int, conv: ConvolutionType = ConvolutionType.STANDARD, flags: int = 0):
        self.D = int(D)
        self.flags = flags
        self._h = None
        self.csm = None
        self.dcw = None
        self.ncoils = 0
        self.matrix_size = None
        self.domain_dims = None
        self.codomain_dims = None
        self.weight = 1.0
        self._traj = None
        self.num_samples = 0
        self.num_frames = 0

    def __del__(self):
        if getattr(self, "_h", None) is not None and lib is not None:
            lib.gb_sense_destroy(self._h)
            self._h = None

    # setup(matrix_size, matrix_size_os, W)  (.cu:64-69)
    def setup(self, matrix_size: Sequence[int], matrix_size_os: Sequence[int], W: float):
        if self._h is not None:
            lib.gb_sense_destroy(self._h)
            self._h = None
        h = ctypes.c_void_p()
        check(lib.gb_sense_create(self.D, _u64(matrix_size), _u64(matrix_size_os), ctypes.c_float(W),
                                  self.flags, ctypes.byref(h)))
        self._h = h
        self.matrix_size = tuple(int(n) for n in matrix_size)
        self.matrix_size_os = tuple(int(m) for m in matrix_size_os)
        self.W = float(W)
        if self.csm is not None:
            check(lib.gb_sense_set_csm(self._h, _ptr(self.csm), self.ncoils))
        if self.dcw is not None:
            check(lib.gb_sense_set_dcw(self._h, _ptr(self.dcw)))

    def set_domain_dimensions(self, dims):
        self.domain_dims = tuple(dims)

    def set_codomain_dimensions(self, dims):
        self.codomain_dims = tuple(dims)

    def get_domain_dimensions(self):
        return self.domain_dims

    def get_codomain_dimensions(self):
        return self.codomain_dims

    def set_weight(self, w: float):
        self.weight = float(w)

    def get_weight(self) -> float:
        return self.weight

    # senseOperator::set_csm (senseOperator.h:26-35)
    def set_csm(self, csm: torch.Tensor):
        _check_tensor(csm, torch.complex64, "csm")
        if csm.dim() != self.D + 1:
            raise ValueError("Error: senseOperator::set_csm : unexpected csm dimensionality")
        self.csm = csm
        self.ncoils = csm.shape[0]
        if self._h is not None:
            check(lib.gb_sense_set_csm(self._h, _ptr(csm), self.ncoils))

    def get_number_of_coils(self) -> int:
        return self.ncoils

    def get_csm(self):
        return self.csm

    def set_dcw(self, dcw: Optional[torch.Tensor]):
        if dcw is not None:
            _check_tensor(dcw, torch.float32, "dcw")
        self.dcw = dcw
        if self._h is not None:
            check(lib.gb_sense_set_dcw(self._h, _ptr(dcw)))

    # preprocess(trajectory)  (.cu:71-84)
    def preprocess(self, trajectory: torch.Tensor, num_frames: int = 1,
                   frame_offsets: Optional[Sequence[int]] = None):
        if trajectory is None:
            raise ValueError("cuNonCartesianSenseOperator: cannot preprocess 0x0 trajectory.")
        if self._h is None:
            raise RuntimeError("setup() must be called before preprocess()")
        _check_tensor(trajectory, torch.float32, "trajectory")
        M = trajectory.numel() // self.D
        if frame_offsets is not None:
            num_frames = len(frame_offsets) - 1
            offs = _u64(frame_offsets)
        else:
            offs = None
        check(lib.gb_sense_preprocess(self._h, _ptr(trajectory), M, int(num_frames), offs, _stream()))
        self._traj = trajectory
        self.num_samples = M
        self.num_frames = int(num_frames)
        self.frame_offsets = list(frame_offsets) if frame_offsets is not None else None

    def _check_io(self, image: torch.Tensor, samples: torch.Tensor):
        _check_tensor(image, torch.complex64, "image")
        _check_tensor(samples, torch.complex64, "samples")
        n = 1
        for v in self.matrix_size:
            n *= v
        if image.numel() != n * self.num_frames:
            raise ValueError("input/output arrays do not match specified domain/codomains")
        if samples.numel() != self.num_samples * self.ncoils:
            raise ValueError("input/output arrays do not match specified domain/codomains")

    def mult_M(self, inp: torch.Tensor, out: torch.Tensor, accumulate: bool = False):
        self._check_io(inp, out)
        check(lib.gb_sense_mult_M(self._h, _ptr(inp), _ptr(out), int(bool(accumulate)), _stream()))

    def mult_MH(self, inp: torch.Tensor, out: torch.Tensor, accumulate: bool = False):
        self._check_io(out, inp)
        check(lib.gb_sense_mult_MH(self._h, _ptr(inp), _ptr(out), int(bool(accumulate)), _stream()))

    def mult_MH_M(self, inp: torch.Tensor, out: torch.Tensor, accumulate: bool = False):
        _check_tensor(inp, torch.complex64, "in")
        _check_tensor(out, torch.complex64, "out")
        check(lib.gb_sense_mult_MH_M(self._h, _ptr(inp), _ptr(out), int(bool(accumulate)), _stream()))

    def autotune(self):
        """Time candidate tilings for this trajectory and coil count; keep the fastest."""
        check(lib.gb_sense_autotune(self._h, _stream()))

    def get_plan(self) -> cuNFFT_plan:
        h = ctypes.c_void_p()
        check(lib.gb_sense_get_nufft_plan(self._h, ctypes.byref(h)))
        p = cuNFFT_plan(self.matrix_size, self.matrix_size_os, self.W, _handle=h)
        p.num_samples = self.num_samples
        p.num_frames = self.num_frames
        p._keep = [self]
        return p
