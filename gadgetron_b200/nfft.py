"""Python mirror of Gadgetron's GPU NFFT plan interface over the C ABI.

Mirrors ``NFFT<cuNDArray,float,D>::make_plan`` and ``NFFT_plan`` /
``cuNFFT_impl`` (toolboxes/nfft/NFFT.h:54-175, toolboxes/nfft/gpu/cuNFFT.h:52-121):
the same method names, argument meanings and error behaviour (errors raise).

Arrays are CUDA ``torch`` tensors (torch supplies device memory and the
current stream; all arithmetic runs in libgadgetron_b200.so).  Shapes follow
the reference's x-fastest layout read in C order:
  image        (..., N_{D-1}, ..., N_0)       complex64   (leading dims: batches, frames)
  oversampled  (..., mos_{D-1}, ..., mos_0)   complex64
  samples      (batches, M_total)             complex64
  trajectory   (M_total, D)                   float32 in [-1/2, 1/2]
  dcw          (M_total,)                     float32
"""
from __future__ import annotations

import ctypes
import enum
from typing import Optional, Sequence

import torch

from ._lib import check, lib


class NFFT_comp_mode(enum.IntEnum):
    FORWARDS_C2NC = 0
    FORWARDS_NC2C = 1
    BACKWARDS_C2NC = 2
    BACKWARDS_NC2C = 3


class NFFT_prep_mode(enum.IntEnum):
    C2NC = 0
    NC2C = 1
    ALL = 2


class NFFT_conv_mode(enum.IntEnum):
    C2NC = 0
    NC2C = 1


class NFFT_fft_mode(enum.IntEnum):
    FORWARDS = 0
    BACKWARDS = 1


class ConvolutionType(enum.IntEnum):
    """Accepted for interface compatibility (cuGriddingConvolution.h:13-18);
    every type runs the same tiled gridding, which is deterministic like
    STANDARD."""
    STANDARD = 0
    ATOMIC = 1
    SPARSE_MATRIX = 2


FLAG_COMPENSATED = 0x1
FLAG_AUTOTUNE = 0x2
FLAG_REFERENCE_FOLD = 0x4


def _u64(vals):
    arr = (ctypes.c_uint64 * len(vals))(*[int(v) for v in vals])
    return arr


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _check_tensor(t: torch.Tensor, dtype, name: str):
    if not isinstance(t, torch.Tensor):
        raise TypeError("%s must be a torch.Tensor" % name)
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor" % name)
    if t.dtype != dtype:
        raise TypeError("%s must have dtype %s, got %s" % (name, dtype, t.dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if t.is_conj() or t.is_neg():
        # a lazy conjugate/negation view: the memory holds the unconjugated
        # values, which is what the library would read
        raise ValueError("%s is a lazy conj/neg view; call resolve_conj()/resolve_neg() first" % name)


class cuNFFT_plan:
    """NFFT_plan<cuNDArray, float, D> on B200."""

    def __init__(self, matrix_size: Sequence[int], matrix_size_os: Sequence[int], W: float,
                 flags: int = 0, _handle=None):
        self.D = len(matrix_size)
        if len(matrix_size_os) != self.D:
            raise ValueError("matrix_size and matrix_size_os must have the same length")
        self.matrix_size = tuple(int(n) for n in matrix_size)
        self.matrix_size_os = tuple(int(m) for m in matrix_size_os)
        self.W = float(W)
        self._owned = _handle is None
        if _handle is None:
            h = ctypes.c_void_p()
            check(lib.gb_nufft_plan_create(self.D, _u64(self.matrix_size), _u64(self.matrix_size_os),
                                           ctypes.c_float(W), flags, ctypes.byref(h)))
            self._h = h
        else:
            self._h = _handle
        self.num_samples = 0
        self.num_frames = 0
        self.frame_offsets = None
        self._keep = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and self._owned and lib is not None:
            lib.gb_nufft_plan_destroy(h)
            self._h = None

    # -- setup queries (NFFT.h:135-151)
    def get_matrix_size(self):
        return self.matrix_size

    def get_matrix_size_os(self):
        return self.matrix_size_os

    def get_W(self):
        return self.W

    def get_tiling(self):
        tile = (ctypes.c_int * 3)()
        cg = ctypes.c_int()
        check(lib.gb_nufft_get_tiling(self._h, tile, ctypes.byref(cg)))
        return tuple(tile[: self.D]), cg.value

    def device_errors(self) -> int:
        """Error bits set on the device by kernels whose bounded waits ran out
        (0: none); reading clears them."""
        bits = ctypes.c_uint32()
        check(lib.gb_nufft_device_errors(self._h, ctypes.byref(bits), _stream()))
        return bits.value

    def autotune(self, num_batches: int = 1):
        """Time candidate tilings on this trajectory and keep the fastest."""
        check(lib.gb_nufft_autotune(self._h, int(num_batches), _stream()))

    def time_normal_convolutions(self, num_batches: int, dcw: Optional[torch.Tensor] = None, reps: int = 20,
                                 flush: Optional[torch.Tensor] = None):
        """Diagnostic: ms per launch of the gridding and the degridding that
        E^H E runs for num_batches batches (cold L2 when a flush buffer is
        given).  Returns (ms_grid, ms_degrid)."""
        g, d = ctypes.c_float(), ctypes.c_float()
        fb = 0 if flush is None else flush.numel() * flush.element_size()
        check(lib.gb_nufft_time_normal_convolutions(self._h, int(num_batches), _ptr(dcw), int(reps), _ptr(flush),
                                                    int(fb), ctypes.byref(g), ctypes.byref(d), _stream()))
        return float(g.value), float(d.value)

    def set_tiling(self, tile: Sequence[int], coil_group: int):
        t = (ctypes.c_int * 3)(*(list(tile) + [1] * (3 - len(tile))))
        check(lib.gb_nufft_set_tiling(self._h, t, int(coil_group)))

    def set_grid_schedule(self, schedule: int):
        """Gridding schedule of the normal operator: 0 by launch depth, 1 one
        CTA per work item, 2 one persistent work-queue launch (same results)."""
        check(lib.gb_nufft_set_grid_schedule(self._h, int(schedule)))

    def get_grid_schedule(self) -> int:
        v = ctypes.c_int()
        check(lib.gb_nufft_get_grid_schedule(self._h, ctypes.byref(v)))
        return v.value

    # -- NFFT_plan::preprocess (NFFT.h:67-68)
    def preprocess(self, trajectory: torch.Tensor, mode: NFFT_prep_mode = NFFT_prep_mode.ALL,
                   num_frames: int = 1, frame_offsets: Optional[Sequence[int]] = None):
        _check_tensor(trajectory, torch.float32, "trajectory")
        if trajectory.shape[-1] != self.D:
            raise ValueError("trajectory must end in a dimension of size D=%d" % self.D)
        M = trajectory.numel() // self.D
        if frame_offsets is not None:
            num_frames = len(frame_offsets) - 1
            offs = _u64(frame_offsets)
        else:
            if trajectory.dim() == 3:
                num_frames = trajectory.shape[0]
            offs = None
        check(lib.gb_nufft_preprocess(self._h, _ptr(trajectory), M, int(num_frames), offs, int(mode),
                                      _stream()))
        self.num_samples = M
        self.num_frames = int(num_frames)
        self.frame_offsets = list(frame_offsets) if frame_offsets is not None else None
        self._keep = [trajectory]

    def _image_info(self, image: torch.Tensor):
        """Returns (oversampled, batches) for an image-side array."""
        n_img = 1
        for v in self.matrix_size:
            n_img *= v
        n_os = 1
        for v in self.matrix_size_os:
            n_os *= v
        tail = tuple(image.shape[-self.D:]) if image.dim() >= self.D else ()
        if tail == tuple(reversed(self.matrix_size_os)) and tail != tuple(reversed(self.matrix_size)):
            per = n_os
            os_ = True
        elif tail == tuple(reversed(self.matrix_size)):
            per = n_img
            os_ = False
        else:
            raise ValueError("image dimensions match neither the matrix size nor the oversampled size")
        per_frames = per * max(1, self.num_frames)
        if image.numel() % per_frames:
            raise ValueError("image size is not a multiple of (matrix size x frames)")
        return os_, image.numel() // per_frames

    # -- NFFT_plan::compute (NFFT.h:77-78)
    def compute(self, inp: torch.Tensor, out: torch.Tensor, dcw: Optional[torch.Tensor],
                mode: NFFT_comp_mode):
        _check_tensor(inp, torch.complex64, "in")
        _check_tensor(out, torch.complex64, "out")
        if dcw is not None:
            _check_tensor(dcw, torch.float32, "dcw")
            if dcw.numel() != self.num_samples:
                raise ValueError("dcw must hold one weight per sample")
        image = inp if mode in (NFFT_comp_mode.FORWARDS_C2NC, NFFT_comp_mode.BACKWARDS_C2NC) else out
        samples = out if image is inp else inp
        if self.num_samples == 0:   # let the library report the missing preprocess
            check(lib.gb_nufft_compute(self._h, _ptr(inp), _ptr(out), _ptr(dcw), int(mode), 1, 0, _stream()))
        os_, nb = self._image_info(image)
        if samples.numel() != nb * self.num_samples:
            raise ValueError("The number of samples is not a multiple of #samples/frame x #frames")
        check(lib.gb_nufft_compute(self._h, _ptr(inp), _ptr(out), _ptr(dcw), int(mode), nb, int(os_),
                                   _stream()))

    # -- NFFT_plan::mult_MH_M (NFFT.h:88-90)
    def mult_MH_M(self, inp: torch.Tensor, out: torch.Tensor, dcw: Optional[torch.Tensor] = None):
        _check_tensor(inp, torch.complex64, "in")
        _check_tensor(out, torch.complex64, "out")
        os_, nb = self._image_info(inp)
        if os_:
            raise ValueError("mult_MH_M takes images of the matrix size")
        if out.numel() != inp.numel():
            raise ValueError("in and out must have the same size")
        if dcw is not None:
            _check_tensor(dcw, torch.float32, "dcw")
        check(lib.gb_nufft_mult_MH_M(self._h, _ptr(inp), _ptr(out), _ptr(dcw), nb, _stream()))

    # -- NFFT_plan::convolve (NFFT.h:103-105)
    def convolve(self, inp: torch.Tensor, out: torch.Tensor, mode: NFFT_conv_mode, accumulate: bool = False):
        _check_tensor(inp, torch.complex64, "in")
        _check_tensor(out, torch.complex64, "out")
        image = inp if mode == NFFT_conv_mode.C2NC else out
        os_, nb = self._image_info(image)
        if not os_:
            raise ValueError("Image dimensions mismatch.")
        check(lib.gb_nufft_convolve(self._h, _ptr(inp), _ptr(out), int(mode), int(bool(accumulate)), nb,
                                    _stream()))

    # -- cuNFFT_impl::fft (cuNFFT.cu:58-70)
    def fft(self, data: torch.Tensor, mode: NFFT_fft_mode, do_scale: bool = True):
        _check_tensor(data, torch.complex64, "data")
        n_os = 1
        for v in self.matrix_size_os:
            n_os *= v
        if data.numel() % n_os:
            raise ValueError("fft: array is not a multiple of the oversampled size")
        check(lib.gb_nufft_fft(self._h, _ptr(data), int(mode), int(bool(do_scale)), data.numel() // n_os,
                               _stream()))

    # -- cuNFFT_impl::deapodize (cuNFFT.cu:74-92)
    def deapodize(self, image: torch.Tensor, fourier_domain: bool = False):
        _check_tensor(image, torch.complex64, "image")
        os_, _ = self._image_info(image)
        if not os_:
            raise ValueError("Error: cuNFFT_impl::deapodize: ERROR: oversampled image not provided as input.")
        n_os = 1
        for v in self.matrix_size_os:
            n_os *= v
        check(lib.gb_nufft_deapodize(self._h, _ptr(image), int(bool(fourier_domain)), image.numel() // n_os,
                                     _stream()))

    # -- trajectory gradient (new surface)
    def traj_grad(self, image: torch.Tensor, weights: torch.Tensor, dcw: Optional[torch.Tensor] = None,
                  out: Optional[torch.Tensor] = None) -> torch.Tensor:
        _check_tensor(image, torch.complex64, "image")
        _check_tensor(weights, torch.complex64, "weights")
        os_, nb = self._image_info(image)
        if os_:
            raise ValueError("traj_grad takes images of the matrix size")
        if out is None:
            out = torch.empty((self.num_samples, self.D), dtype=torch.float32, device=image.device)
        check(lib.gb_nufft_traj_grad(self._h, _ptr(image), _ptr(weights), _ptr(dcw), _ptr(out), nb, _stream()))
        return out

    def traj_grad_from_grid(self, grid: torch.Tensor, weights: torch.Tensor,
                            out: Optional[torch.Tensor] = None) -> torch.Tensor:
        _check_tensor(grid, torch.complex64, "grid")
        _check_tensor(weights, torch.complex64, "weights")
        os_, nb = self._image_info(grid)
        if not os_:
            raise ValueError("traj_grad_from_grid takes an oversampled grid")
        if out is None:
            out = torch.empty((self.num_samples, self.D), dtype=torch.float32, device=grid.device)
        check(lib.gb_nufft_traj_grad_from_grid(self._h, _ptr(grid), _ptr(weights), _ptr(out), nb, _stream()))
        return out


class NFFT:
    """NFFT<cuNDArray, float, D>::make_plan (cuNFFT.h:113-121)."""

    @staticmethod
    def make_plan(matrix_size, matrix_size_os, W, conv: ConvolutionType = ConvolutionType.STANDARD,
                  flags: int = 0) -> cuNFFT_plan:
        return cuNFFT_plan(matrix_size, matrix_size_os, W, flags)
