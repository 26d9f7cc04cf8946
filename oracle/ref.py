"""Test infrastructure: numpy-facing binding of oracle/_ref/libgbref.so, the
reference's own GPU path (cuNFFT_impl<float,D,STANDARD>,
cuNonCartesianSenseOperator, cuCgSolver) built from its sources by
oracle/build_ref.py.  Only tests, smoke() and bench.py's reference legs use
it, as the parity anchor for the product.

Array conventions match the product's Python API (numpy C order, so the last
axis is the reference's fastest dimension x):
  traj     (F*M, D) float32, coordinates in [-0.5, 0.5]
  image    (B, F, *N) complex64   == reference dims [N..., F, B]
  samples  (B, F*M) complex64     == reference dims [M, F, B]
  dcw      (F*M,) float32         == reference dims [M, F]
  csm      (C, *N) complex64      == reference dims [N..., C]
  SENSE data (C, F*M) complex64   == reference dims [M*F, C]
N and mos are given x-first, as the reference's vector_td lists them.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgbref.so")

COMP_MODES = {"FORWARDS_C2NC": 0, "FORWARDS_NC2C": 1, "BACKWARDS_C2NC": 2, "BACKWARDS_NC2C": 3}

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference build missing: run python oracle/build_ref.py (needs the reference sources)")
        L = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        vp, fp, i, u64, f = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_uint64, ctypes.c_float
        L.gbref_last_error.restype = ctypes.c_char_p
        L.gbref_nfft_compute.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, vp, fp, i, u64, i, i]
        L.gbref_nfft_mult_MH_M.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, vp, fp, u64]
        L.gbref_nfft_convolve.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, vp, i, u64, i]
        L.gbref_nfft_fft_deapodize.argtypes = [i, u64p, u64p, f, vp, u64, i, i]
        L.gbref_sense_mult.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, u64, fp, vp, vp, i]
        L.gbref_cg_sense.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, u64, fp, vp, vp, i, f, vp,
                                     ctypes.POINTER(ctypes.c_int)]
        fpp = ctypes.POINTER(ctypes.c_float)
        L.gbref_time_cg_sense.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, u64, fp, vp, i, i, fpp]
        L.gbref_time_nfft.argtypes = [i, u64p, u64p, f, fp, u64, u64, vp, fp, u64, i, fpp, fpp, fpp]
        for name in ("gbref_time_cg_sense", "gbref_time_nfft", "gbref_nfft_compute", "gbref_nfft_mult_MH_M", "gbref_nfft_convolve",
                     "gbref_nfft_fft_deapodize", "gbref_sense_mult", "gbref_cg_sense"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _u64(v):
    return (ctypes.c_uint64 * len(v))(*[int(x) for x in v])


def _f32(a):
    a = np.ascontiguousarray(a, np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _c64(a):
    return np.ascontiguousarray(a, np.complex64)


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + lib().gbref_last_error().decode(errors="replace"))


def _traj(traj, D):
    t = np.ascontiguousarray(traj, np.float32).reshape(-1, D)
    return t, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def nfft_compute(N, mos, W, traj, frames, x, dcw, mode, batches=1, oversampled_image=False, conv_type=0):
    """cuNFFT_plan::compute (nfft/NFFT.hpp:105-203) on a fresh plan preprocessed
    with the trajectory, exactly as its callers run it."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    m = COMP_MODES[mode] if isinstance(mode, str) else int(mode)
    img_shape = (batches, frames) + tuple(reversed(mos if oversampled_image else N))
    smp_shape = (batches, frames * M)
    c2nc = m in (0, 2)
    xin = _c64(x)
    out = np.empty(smp_shape if c2nc else img_shape, np.complex64)
    keep = None
    dp = None
    if dcw is not None:
        keep, dp = _f32(dcw)
    _check(lib().gbref_nfft_compute(D, _u64(N), _u64(mos), float(W), tp, M, frames, xin.ctypes.data,
                                    out.ctypes.data, dp, m, batches, int(oversampled_image), int(conv_type)))
    return out


def nfft_mult_MH_M(N, mos, W, traj, frames, x, dcw, batches=1):
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    xin = _c64(x)
    out = np.empty((batches, frames) + tuple(reversed(N)), np.complex64)
    keep, dp = (None, None) if dcw is None else _f32(dcw)
    _check(lib().gbref_nfft_mult_MH_M(D, _u64(N), _u64(mos), float(W), tp, M, frames, xin.ctypes.data,
                                      out.ctypes.data, dp, batches))
    return out


def nfft_convolve(N, mos, W, traj, frames, x, conv, batches=1, out=None, accumulate=False):
    """Standalone convolution (NFFT.h:103-105); conv 'C2NC' (oversampled grid
    -> samples) or 'NC2C' (samples -> oversampled grid)."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    c = 0 if conv == "C2NC" else 1
    shape = (batches, frames * M) if c == 0 else (batches, frames) + tuple(reversed(mos))
    res = np.zeros(shape, np.complex64) if out is None else np.array(out, np.complex64, copy=True)
    xin = _c64(x)
    _check(lib().gbref_nfft_convolve(D, _u64(N), _u64(mos), float(W), tp, M, frames, xin.ctypes.data,
                                     res.ctypes.data, c, batches, int(accumulate)))
    return res


def nfft_fft(N, mos, W, data, forwards=True, do_scale=True):
    """cuNFFT_impl::fft (cuNFFT.cu:58-70) in place on (FB, *mos) data."""
    d = np.array(data, np.complex64, copy=True)
    FB = d.size // int(np.prod(mos))
    _check(lib().gbref_nfft_fft_deapodize(len(N), _u64(N), _u64(mos), float(W), d.ctypes.data, FB,
                                          0 if forwards else 1, int(do_scale)))
    return d


def nfft_deapodize(N, mos, W, data, fourier_domain=False):
    """cuNFFT_impl::deapodize (cuNFFT.cu:74-92) in place on (FB, *mos) data."""
    d = np.array(data, np.complex64, copy=True)
    FB = d.size // int(np.prod(mos))
    _check(lib().gbref_nfft_fft_deapodize(len(N), _u64(N), _u64(mos), float(W), d.ctypes.data, FB,
                                          3 if fourier_domain else 2, 0))
    return d


def sense_mult(N, mos, W, traj, frames, csm, dcw, x, adjoint=False):
    """cuNonCartesianSenseOperator::mult_M / mult_MH (.cu:14-63)."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    csm = _c64(csm)
    C = csm.shape[0]
    keep, dp = (None, None) if dcw is None else _f32(dcw)
    xin = _c64(x)
    out = np.empty((frames,) + tuple(reversed(N)) if adjoint else (C, frames * M), np.complex64)
    _check(lib().gbref_sense_mult(D, _u64(N), _u64(mos), float(W), tp, M, frames, csm.ctypes.data, C, dp,
                                  xin.ctypes.data, out.ctypes.data, int(adjoint)))
    return out


def cg_sense(N, mos, W, traj, frames, csm, dcw, data, iterations, tc_tolerance=0.0, keep_iterates=False):
    """cuCgSolver<float_complext>::solve (solvers/cgSolver.h:105-390) with a
    cuNonCartesianSenseOperator encoding operator set up as
    gadgets/pmri/gpuCgSenseGadget.cpp:155-199 does (no regulariser, no
    preconditioner).  Returns x, or (x, iterates[k]) with every iterate."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    csm = _c64(csm)
    C = csm.shape[0]
    keep, dp = (None, None) if dcw is None else _f32(dcw)
    d = _c64(data)
    img_shape = (frames,) + tuple(reversed(N))
    x = np.empty(img_shape, np.complex64)
    its = np.empty((max(iterations, 1),) + img_shape, np.complex64) if keep_iterates else None
    ran = ctypes.c_int(0)
    _check(lib().gbref_cg_sense(D, _u64(N), _u64(mos), float(W), tp, M, frames, csm.ctypes.data, C, dp,
                                d.ctypes.data, x.ctypes.data, int(iterations), float(tc_tolerance),
                                None if its is None else its.ctypes.data, ctypes.byref(ran)))
    if keep_iterates:
        return x, its[:ran.value]
    return x


def time_cg_sense(N, mos, W, traj, frames, csm, dcw, data, iterations, reps=5):
    """Device ms of one reference cuCgSolver::solve (tc_tolerance 0) on the
    current GPU, operator preprocessed, inputs resident."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    csm = _c64(csm)
    keep, dp = (None, None) if dcw is None else _f32(dcw)
    d = _c64(data)
    ms = ctypes.c_float(0)
    _check(lib().gbref_time_cg_sense(D, _u64(N), _u64(mos), float(W), tp, M, frames, csm.ctypes.data, csm.shape[0],
                                     dp, d.ctypes.data, int(iterations), int(reps), ctypes.byref(ms)))
    return float(ms.value)


def time_nfft(N, mos, W, traj, frames, img, dcw, batches=1, reps=5):
    """Device ms of the reference's preprocess, compute(FORWARDS_C2NC) and
    compute(BACKWARDS_NC2C, dcw): (fwd, adj, preprocess)."""
    D = len(N)
    t, tp = _traj(traj, D)
    M = t.shape[0] // frames
    x = _c64(img)
    keep, dp = (None, None) if dcw is None else _f32(dcw)
    a, b, c = ctypes.c_float(0), ctypes.c_float(0), ctypes.c_float(0)
    _check(lib().gbref_time_nfft(D, _u64(N), _u64(mos), float(W), tp, M, frames, x.ctypes.data, dp, batches,
                                 int(reps), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return float(a.value), float(b.value), float(c.value)
