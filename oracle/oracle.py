"""CPU oracle for the non-Cartesian NUFFT / CG-SENSE path (test infrastructure).

This module is the checker for the CUDA library in ``gadgetron_b200``.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it; the product never does.

Parity status: pinned against the reference's own outputs.  The reference's
GPU path is built from its sources (oracle/build_ref.py -> oracle/_ref) and
tests/test_ref_parity_gpu.py checks this restatement against it on the same
seeded inputs (NUFFT in 2D and 3D, SENSE operator, CG iterates), besides the
reference's own known-answer test setups, the FP64 direct NDFT and exact
adjointness (tests/test_known_answers.py, tests/test_oracle.py).  In 3D the
reference folds the gridding's padding ring differently from the periodic
fold near z faces; ``OraclePlan(..., reference_fold=True)`` restates that
fold so the 3D adjoint is pinned as well (see nufft_oracle.c).

It restates the reference GPU path (Gadgetron cuNFFT, STANDARD convolution,
cuNonCartesianSenseOperator and cgSolver) on the CPU:

* gridding, degridding and the kernel image of the deapodization filter are in
  ``nufft_oracle.c`` (float kernel weights as the reference computes them,
  double accumulation), loaded here through ctypes;
* the centred FFT follows ``toolboxes/fft/gpu/cuNDFFT.cpp:184-252`` and
  ``toolboxes/fft/gpu/cuNDFFT.cu:6-36``: checkerboard ("timeswitch") before and
  after an unnormalised C2C transform, CUFFT_FORWARD = exp(-i), then a scale
  by 1/sqrt(prod(size)) when ``do_scale``; computed here in complex128;
* the deapodization filter follows ``toolboxes/nfft/gpu/cuNFFT.cu:171-202``:
  kernel image, *unscaled* centred FFT (BACKWARDS for the image-domain
  filter, FORWARDS for the Fourier-domain one), reciprocal;
* ``compute`` follows ``toolboxes/nfft/NFFT.hpp:105-240`` (pad/crop offsets
  ``toolboxes/core/gpu/cuNDArray_utils.cu:213-300``), ``mult_MH_M`` follows
  ``NFFT.hpp:90-102``;
* the SENSE operator follows
  ``toolboxes/mri/pmri/gpu/cuNonCartesianSenseOperator.cu:14-62`` and
  ``toolboxes/mri/pmri/gpu/sense_utilities.cu:7-123``;
* the CG solver follows ``toolboxes/solvers/cgSolver.h:105-390`` with the
  ``relativeResidualTCB`` stop rule of ``toolboxes/solvers/cgCallback.h:56-104``;
  regularisation terms w_i R_i^H R_i follow ``cgSolver.h:355-390``;
* radial trajectories and their Voronoi density compensation weights follow
  ``toolboxes/core/gpu/radial_utilities.cu:18-441``;
* the density compensation estimate follows ``toolboxes/mri/sdc/SDC.hpp:19-80``
  with the Jinc kernel of ``toolboxes/nfft/ConvolutionKernel.hpp:307-397``;
* the SENSE accumulation buffer follows ``toolboxes/mri/pmri/gpu/cuBuffer.cpp:7-166``
  and ``cuSenseBuffer.cpp:18-35``;
* the coil sensitivity estimate follows ``toolboxes/mri/pmri/gpu/b1_map.cu:29-118``
  (RSS normalisation, correlation matrices, 7^D box smoothing, two power
  iterations, coil-0 phase reference);
* the image regulariser follows ``toolboxes/operators/imageOperator.h:27-67``
  and its offset estimate ``toolboxes/operators/gpu/cuImageOperator.h:35-62``;
  the preconditioner weights follow ``gadgets/pmri/gpuCgSenseGadget.cpp:167-176``.

The direct FP64 NDFT (``ndft_forward``/``ndft_adjoint``) is the accuracy
oracle: y_j = dcw_j / sqrt(G) * sum_n x_n exp(-2 pi i k_j.(n - N/2)), G the
number of oversampled grid cells.

Array conventions (numpy, C order, x on the last axis):
  image    [nb, F, *N[::-1]]     complex
  grid     [nb, F, *mos[::-1]]   complex
  samples  [nb, F, M]            complex
  traj     [F, M, D]             float32 in [-1/2, 1/2], component 0 = x
  dcw      [F, M]                float
  csm      [C, *N[::-1]]         complex
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "nufft_oracle.c")
_LIB_PATH = os.path.join(_HERE, "liboracle_nufft.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile nufft_oracle.c with gcc (OpenMP, no FMA contraction)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC)):
        tmp = _LIB_PATH + ".tmp%d" % os.getpid()
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-std=c11", "-D_DEFAULT_SOURCE", _SRC, "-o", tmp, "-lm"]
        subprocess.check_call(cmd)
        os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        f32 = ctypes.c_float
        L.or_bessi0f.restype = f32
        L.or_bessi0f.argtypes = [f32]
        L.or_kb1f.restype = f32
        L.or_kb1f.argtypes = [f32, f32, f32, f32]
        L.or_kb_get_1d.restype = f32
        L.or_kb_get_1d.argtypes = [f32, f32, f32, f32, f32]
        L.or_compute_beta.argtypes = [ctypes.c_int, P, P, f32, P]
        L.or_scale_trajectory.restype = ctypes.c_int
        L.or_scale_trajectory.argtypes = [ctypes.c_int, P, P, f32, P, i64, P]
        L.or_grid_nc2c.argtypes = [ctypes.c_int, P, P, f32, i64, i64, i64, P, P, P, ctypes.c_int]
        L.ho_matrix_create.restype = P
        L.ho_matrix_create.argtypes = [ctypes.c_int, P, P, f32, P, i64]
        L.ho_matrix_destroy.argtypes = [P]
        L.ho_c2nc.argtypes = [P, i64, P, P, ctypes.c_int]
        L.ho_nc2c.argtypes = [P, i64, P, P, ctypes.c_int]
        L.or_grid_nc2c_fold.argtypes = [ctypes.c_int, P, P, f32, i64, i64, i64, P, P, P, ctypes.c_int,
                                        ctypes.c_int]
        L.or_degrid_c2nc.argtypes = [ctypes.c_int, P, P, f32, i64, i64, i64, P, P, P, ctypes.c_int]
        L.or_deapod_kernel_image.argtypes = [ctypes.c_int, P, P, f32, P]
        L.or_ndft_forward.argtypes = [ctypes.c_int, P, ctypes.c_double, i64, i64, P, P, P, P]
        L.or_ndft_adjoint.argtypes = [ctypes.c_int, P, ctypes.c_double, i64, i64, P, P, P, P]
        L.or_num_threads.restype = ctypes.c_int
        L.or_degrid_traj_grad.argtypes = [ctypes.c_int, P, P, f32, i64, i64, i64, P, P, P, P]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _u64(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.uint64))


def num_threads() -> int:
    return int(lib().or_num_threads())


# ---------------------------------------------------------------- kernel ---

def bessi0f(x: float) -> float:
    return float(lib().or_bessi0f(np.float32(x)))


def kb_beta(N, mos, W):
    beta = np.zeros(len(N), np.float32)
    lib().or_compute_beta(len(N), _p(_u64(N)), _p(_u64(mos)), np.float32(W), _p(beta))
    return beta


def kb_get_1d(delta: float, mos_d: int, W: float, beta_d: float) -> float:
    W = np.float32(W)
    return float(lib().or_kb_get_1d(np.float32(delta), np.float32(mos_d),
                                    np.float32(1.0) / W, np.float32(beta_d),
                                    W / np.float32(2.0)))


# -------------------------------------------------------------- centred FFT --

def timeswitch(a: np.ndarray, D: int) -> np.ndarray:
    """Multiply by (-1)^(sum of coordinates) over the last D axes
    (cuNDFFT.cu:6-36)."""
    sign = np.ones(a.shape[-D:], dtype=np.float64)
    for ax in range(D):
        n = a.shape[a.ndim - D + ax]
        s = np.where(np.arange(n) % 2 == 1, -1.0, 1.0)
        shape = [1] * D
        shape[ax] = n
        sign = sign * s.reshape(shape)
    return a * sign


_FFT_WORKERS = 1


def set_fft_workers(n: int):
    """Use scipy.fft (pocketfft) with n threads for the oracle's FFTs (n > 1),
    as the timed CPU baseline does; numpy's FFT otherwise."""
    global _FFT_WORKERS
    _FFT_WORKERS = int(n)


def centred_fft(a: np.ndarray, D: int, forward: bool, do_scale: bool = True) -> np.ndarray:
    """cuNDFFT::fft / ifft over the last D axes (cuNDFFT.cpp:184-252)."""
    axes = tuple(range(a.ndim - D, a.ndim))
    b = timeswitch(np.asarray(a, dtype=np.complex128), D)
    if _FFT_WORKERS > 1:
        import scipy.fft as sfft
        if forward:
            b = sfft.fftn(b, axes=axes, workers=_FFT_WORKERS)
        else:
            b = sfft.ifftn(b, axes=axes, norm="forward", workers=_FFT_WORKERS)
    elif forward:
        b = np.fft.fftn(b, axes=axes)               # CUFFT_FORWARD, unnormalised
    else:
        b = np.fft.ifftn(b, axes=axes, norm="forward")  # CUFFT_INVERSE, unnormalised
    b = timeswitch(b, D)
    if do_scale:
        G = int(np.prod([a.shape[ax] for ax in axes]))
        b = b / np.sqrt(G)
    return b


# ------------------------------------------------------------ pad / crop ----

def pad(img: np.ndarray, mos, D: int) -> np.ndarray:
    """Centred zero-fill, offset mos/2 - N/2 (cuNDArray_utils.cu:273-300)."""
    N = img.shape[-D:]
    mos_r = tuple(int(m) for m in mos[::-1])
    out = np.zeros(img.shape[:-D] + mos_r, dtype=np.complex128)
    sl = tuple(slice(m // 2 - n // 2, m // 2 - n // 2 + n) for n, m in zip(N, mos_r))
    out[(Ellipsis,) + sl] = img
    return out


def crop(grid: np.ndarray, N, D: int) -> np.ndarray:
    """Centred crop, offset (mos - N) >> 1 (NFFT.hpp:178-181)."""
    mos = grid.shape[-D:]
    N_r = tuple(int(n) for n in N[::-1])
    sl = tuple(slice((m - n) >> 1, ((m - n) >> 1) + n) for n, m in zip(N_r, mos))
    return grid[(Ellipsis,) + sl].copy()


# ------------------------------------------------------------------ plan ----

class OraclePlan:
    """CPU restatement of cuNFFT_impl<float, D, STANDARD>.

    reference_fold=True folds the gridding's padding ring as the reference's
    wrap_image_kernel does (ConvolverNC2C_standard.cuh:394-437), which in 3D
    differs from the periodic fold on cells near a z face (see
    nufft_oracle.c); the default is the periodic fold the product computes.
    """

    def __init__(self, N, mos, W, reference_fold=False):
        self.fold = 1 if reference_fold else 0
        self.D = len(N)
        self.N = tuple(int(n) for n in N)
        self.mos = tuple(int(m) for m in mos)
        self.W = float(np.float32(W))
        self.G = int(np.prod(self.mos))
        if any(m < n for n, m in zip(self.N, self.mos)):
            raise ValueError("oversampled matrix size must be >= matrix size")
        self._scaled = None
        self.M = 0
        self.F = 0
        self._filter = {}

    # NFFT_plan::preprocess -> cuGriddingConvolution::preprocess
    def preprocess(self, traj: np.ndarray):
        traj = np.ascontiguousarray(traj, dtype=np.float32)
        if traj.ndim == 2:
            traj = traj[None]
        F, M, D = traj.shape
        if D != self.D:
            raise ValueError("trajectory dimensionality mismatch")
        scaled = np.empty_like(traj)
        rc = lib().or_scale_trajectory(self.D, _p(_u64(self.N)), _p(_u64(self.mos)),
                                       np.float32(self.W), _p(traj), F * M, _p(scaled))
        if rc != 0:
            raise ValueError("trajectory out of range [-1/2, 1/2]")
        self._scaled = scaled
        self.M, self.F = M, F

    @property
    def scaled_trajectory(self):
        return self._scaled

    def deapodization_filter(self, fourier_domain: bool = False) -> np.ndarray:
        """1 / unscaled centred FFT of the kernel image (cuNFFT.cu:171-202)."""
        if fourier_domain not in self._filter:
            img = np.empty(self.G, np.float32)
            lib().or_deapod_kernel_image(self.D, _p(_u64(self.N)), _p(_u64(self.mos)),
                                         np.float32(self.W), _p(img))
            img = img.reshape(self.mos[::-1]).astype(np.complex128)
            f = centred_fft(img, self.D, forward=fourier_domain, do_scale=False)
            self._filter[fourier_domain] = 1.0 / f
        return self._filter[fourier_domain]

    def _nb(self, arr: np.ndarray, image_like: bool) -> int:
        per = (int(np.prod(arr.shape[-self.D:])) if image_like else self.M) * self.F
        n = arr.size // per
        if n * per != arr.size or n == 0:
            raise ValueError("array size is not a multiple of the plan's frame size")
        return n

    def convolve_c2nc(self, grid: np.ndarray, accumulate_into=None) -> np.ndarray:
        nb = grid.size // (self.G * self.F)
        g = np.ascontiguousarray(grid, dtype=np.complex128).reshape(nb, self.F, self.G)
        out = (np.zeros((nb, self.F, self.M), np.complex128) if accumulate_into is None
               else np.ascontiguousarray(accumulate_into, dtype=np.complex128).copy())
        lib().or_degrid_c2nc(self.D, _p(_u64(self.N)), _p(_u64(self.mos)), np.float32(self.W),
                             self.M, self.F, nb, _p(self._scaled), _p(g), _p(out),
                             0 if accumulate_into is None else 1)
        return out

    def convolve_nc2c(self, samples: np.ndarray, accumulate_into=None) -> np.ndarray:
        nb = samples.size // (self.M * self.F)
        s = np.ascontiguousarray(samples, dtype=np.complex128).reshape(nb, self.F, self.M)
        out = (np.zeros((nb, self.F) + self.mos[::-1], np.complex128) if accumulate_into is None
               else np.ascontiguousarray(accumulate_into, dtype=np.complex128).copy())
        lib().or_grid_nc2c_fold(self.D, _p(_u64(self.N)), _p(_u64(self.mos)), np.float32(self.W),
                                self.M, self.F, nb, _p(self._scaled), _p(s), _p(out),
                                0 if accumulate_into is None else 1, self.fold)
        return out

    def deapodize(self, image: np.ndarray, fourier_domain: bool = False) -> np.ndarray:
        if tuple(image.shape[-self.D:]) != self.mos[::-1]:
            raise ValueError("deapodize: oversampled image not provided as input")
        return image * self.deapodization_filter(fourier_domain)

    def fft(self, data: np.ndarray, forward: bool, do_scale: bool = True) -> np.ndarray:
        return centred_fft(data, self.D, forward, do_scale)

    # NFFT_plan::compute, modes FORWARDS_C2NC / BACKWARDS_NC2C / FORWARDS_NC2C
    def forward_c2nc(self, image: np.ndarray, dcw=None) -> np.ndarray:
        img = np.asarray(image, dtype=np.complex128)
        if tuple(img.shape[-self.D:]) != self.mos[::-1]:
            img = pad(img, self.mos, self.D)
        nb = img.size // (self.G * self.F)
        img = img.reshape((nb, self.F) + self.mos[::-1])
        img = self.deapodize(img)
        img = self.fft(img, forward=True)
        out = self.convolve_c2nc(img)
        if dcw is not None:
            out = out * np.asarray(dcw, np.float64).reshape(1, self.F, self.M)
        return out

    def backwards_nc2c(self, samples: np.ndarray, dcw=None, oversampled_out=False) -> np.ndarray:
        s = np.asarray(samples, dtype=np.complex128)
        nb = s.size // (self.M * self.F)
        s = s.reshape(nb, self.F, self.M)
        if dcw is not None:
            s = s * np.asarray(dcw, np.float64).reshape(1, self.F, self.M)
        img = self.convolve_nc2c(s)
        img = self.fft(img, forward=False)
        img = self.deapodize(img)
        return img if oversampled_out else crop(img, self.N, self.D)

    def forwards_nc2c(self, samples: np.ndarray, dcw=None, oversampled_out=False) -> np.ndarray:
        s = np.asarray(samples, dtype=np.complex128)
        nb = s.size // (self.M * self.F)
        s = s.reshape(nb, self.F, self.M)
        if dcw is not None:
            s = s * np.asarray(dcw, np.float64).reshape(1, self.F, self.M)
        img = self.convolve_nc2c(s)
        img = self.fft(img, forward=True)
        img = self.deapodize(img, fourier_domain=True)
        return img if oversampled_out else crop(img, self.N, self.D)

    def mult_MH_M(self, image: np.ndarray, dcw=None) -> np.ndarray:
        return self.backwards_nc2c(self.forward_c2nc(image, dcw), dcw)

    def forward_grid(self, image: np.ndarray) -> np.ndarray:
        """The oversampled k-space grid the forward NUFFT degrids from."""
        img = np.asarray(image, dtype=np.complex128)
        if tuple(img.shape[-self.D:]) != self.mos[::-1]:
            img = pad(img, self.mos, self.D)
        nb = img.size // (self.G * self.F)
        img = img.reshape((nb, self.F) + self.mos[::-1])
        return self.fft(self.deapodize(img), forward=True)

    def traj_grad_from_grid(self, grid: np.ndarray, weights: np.ndarray) -> np.ndarray:
        """out[j, d] = sum_b Re(weights[b, j] * d(degrid(grid))[b, j] / d k[j, d]),
        the derivative of the taps' weights of or_degrid_c2nc (new surface; the
        reference has no trajectory derivative)."""
        nb = grid.size // (self.G * self.F)
        g = np.ascontiguousarray(grid, dtype=np.complex128).reshape(nb, self.F, self.G)
        w = np.ascontiguousarray(weights, dtype=np.complex128).reshape(nb, self.F, self.M)
        out = np.zeros((self.F * self.M, self.D), np.float64)
        lib().or_degrid_traj_grad(self.D, _p(_u64(self.N)), _p(_u64(self.mos)), np.float32(self.W),
                                  self.M, self.F, nb, _p(self._scaled), _p(g), _p(w), _p(out))
        return out

    def traj_grad_forward(self, image: np.ndarray, weights: np.ndarray, dcw=None) -> np.ndarray:
        """Gradient of the forward NUFFT (FORWARDS_C2NC, dcw on the output)
        with respect to the trajectory, contracted with complex weights."""
        w = np.asarray(weights, np.complex128).reshape(-1, self.F, self.M)
        if dcw is not None:
            w = w * np.asarray(dcw, np.float64).reshape(1, self.F, self.M)
        return self.traj_grad_from_grid(self.forward_grid(image), w)


# ------------------------------------------- reference CPU path (float) ------

class HoSenseFloat:
    """The reference's CPU reconstruction path in its own float arithmetic,
    for the timed CPU baseline: gridding by the per-sample convolution matrix
    and its transpose of hoGriddingConvolution (ho_matrix_* in
    nufft_oracle.c, complext<float> sums, OpenMP over coils), the centred FFT
    in complex64 (pocketfft through scipy.fft with every host thread, standing
    in for the FFTW the reference links), deapodization, csm multiply and the
    cgSolver iteration (cgSolver.h:105-390) in complex64 with float dots.
    Same operator as OracleSense: E = D^(1/2) NUFFT S."""

    def __init__(self, N, mos, W, traj, csm, dcw, workers=None):
        import scipy.fft as sfft
        self._fft = sfft
        self.D = len(N)
        self.N = tuple(int(n) for n in N)
        self.mos = tuple(int(m) for m in mos)
        self.W = float(np.float32(W))
        self.workers = workers or (os.cpu_count() or 1)
        traj = np.ascontiguousarray(traj, np.float32).reshape(-1, self.D)
        self.M = traj.shape[0]
        self.G = int(np.prod(self.mos))
        self._h = lib().ho_matrix_create(self.D, _p(_u64(self.N)), _p(_u64(self.mos)), np.float32(self.W),
                                         _p(traj), self.M)
        plan = OraclePlan(N, mos, W)
        self.deap = plan.deapodization_filter(False).astype(np.complex64)
        self.csm = np.ascontiguousarray(csm, np.complex64)
        self.C = self.csm.shape[0]
        self.dcw = np.ascontiguousarray(dcw, np.float32).reshape(1, -1)
        self.scale = np.float32(1.0 / np.sqrt(self.G))
        ax = tuple(range(-self.D, 0))
        self._axes = ax

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ho_matrix_destroy(self._h)
            self._h = None

    def _cfft(self, a, forward):
        f = self._fft
        a = f.ifftshift(a, axes=self._axes)
        a = (f.fftn if forward else f.ifftn)(a, axes=self._axes, workers=self.workers,
                                             norm="ortho", overwrite_x=True)
        return f.fftshift(a, axes=self._axes).astype(np.complex64, copy=False)

    def _pad(self, img):
        out = np.zeros((img.shape[0],) + self.mos[::-1], np.complex64)
        sl = tuple(slice((m - n) // 2, (m - n) // 2 + n) for n, m in zip(self.N[::-1], self.mos[::-1]))
        out[(slice(None),) + sl] = img
        return out

    def _crop(self, grid):
        sl = tuple(slice((m - n) // 2, (m - n) // 2 + n) for n, m in zip(self.N[::-1], self.mos[::-1]))
        return np.ascontiguousarray(grid[(slice(None),) + sl])

    def mult_M(self, x):
        """x [*N] -> samples [C, M]."""
        g = self._pad(self.csm * x[None])
        g *= self.deap
        g = self._cfft(g, True)
        y = np.empty((self.C, self.M), np.complex64)
        lib().ho_c2nc(self._h, self.C, _p(g), _p(y), 0)
        y *= self.dcw
        return y

    def mult_MH(self, y):
        """samples [C, M] -> image [*N]."""
        ys = np.ascontiguousarray(y * self.dcw, np.complex64)
        g = np.empty((self.C,) + self.mos[::-1], np.complex64)
        lib().ho_nc2c(self._h, self.C, _p(ys), _p(g), 0)
        g = self._cfft(g, False)
        g *= self.deap
        return np.sum(self._crop(g) * np.conj(self.csm), axis=0)

    def mult_MH_M(self, x):
        return self.mult_MH(self.mult_M(x))

    def cg(self, d, iterations, snapshot=None):
        """cgSolver iteration in complex64 (tc_tolerance 0).  Returns a
        generator that yields after every iteration, so a caller can time
        single iterations; x is in self.x."""
        rhs = self.mult_MH(d)
        self.x = np.zeros_like(rhs)
        r = rhs.copy()
        p = r.copy()
        rq = np.float32(np.real(np.vdot(r, r)))
        for _ in range(iterations):
            q = self.mult_MH_M(p)
            alpha = np.complex64(rq / np.vdot(p, q))
            self.x += alpha * p
            r -= alpha * q
            rq2 = np.float32(np.real(np.vdot(r, r)))
            p = p * np.float32(rq2 / rq) + r
            rq = rq2
            yield self.x


# --------------------------------------------------------------- SENSE ------

class OracleSense:
    """CPU restatement of cuNonCartesianSenseOperator<float, D>."""

    def __init__(self, plan: OraclePlan, csm: np.ndarray, dcw=None):
        self.plan = plan
        self.csm = np.asarray(csm, np.complex128)
        self.dcw = None if dcw is None else np.asarray(dcw, np.float64)

    def mult_M(self, x: np.ndarray) -> np.ndarray:
        # x [F, *N] -> coil images [C, F, *N] (sense_utilities.cu:7-18)
        D = self.plan.D
        coil = self.csm[:, None] * np.asarray(x, np.complex128)[None]
        return self.plan.forward_c2nc(coil, self.dcw)

    def mult_MH(self, y: np.ndarray) -> np.ndarray:
        img = self.plan.backwards_nc2c(y, self.dcw)       # [C, F, *N]
        return np.sum(img * np.conj(self.csm)[:, None], axis=0)  # sense_utilities.cu:66-78

    def mult_MH_M(self, x: np.ndarray) -> np.ndarray:
        return self.mult_MH(self.mult_M(x))


def image_operator_compute(reg_image: np.ndarray, offset_estimation: bool = True):
    """imageOperator::compute (imageOperator.h:27-45) with the offset estimate
    of cuImageOperator::estimate_offset (cuImageOperator.h:35-62), in float32
    as the reference computes it.  Returns (image, offset): image =
    1 / (|reg * n / asum(reg)| + offset), asum = sum |re| + |im| (Scasum);
    offset = (k + 1) * max / 50000 with k the first 50000-bin histogram bin
    of image / max at which the cumulative count reaches 1% of the elements."""
    z = np.asarray(reg_image, np.complex64).ravel()
    n = z.size
    asum = float(np.sum(np.abs(z.real).astype(np.float64) + np.abs(z.imag).astype(np.float64)))
    scale = np.float32(np.float32(n) / np.float32(asum))
    re = (z.real * scale).astype(np.float32)
    im = (z.imag * scale).astype(np.float32)
    img = np.sqrt((re * re).astype(np.float32) + (im * im).astype(np.float32)).astype(np.float32)
    offset = np.float32(0.0)
    if offset_estimation:
        gran = 50000
        mx = np.float32(img.max())
        bins = np.minimum(np.floor((img / mx) * np.float32(gran)).astype(np.int64), gran - 1)
        hist = np.bincount(bins, minlength=gran)
        target = int(np.float32(0.01) * np.float32(n))
        cumsum, counter = 0, 0
        while cumsum < target:
            cumsum += int(hist[counter])
            counter += 1
        offset = np.float32(np.float32(counter + 1) * mx / np.float32(gran))
    if offset > 0:
        img = (img + offset).astype(np.float32)
    img = (np.float32(1.0) / img).astype(np.float32)
    return img.reshape(np.shape(reg_image)), float(offset)


def sense_precond_weights(csm: np.ndarray, reg_image=None, kappa: float = 0.0) -> np.ndarray:
    """Diagonal preconditioner of gpuCgSenseGadget.cpp:167-176:
    1 / sqrt(sum_c |csm_c|^2 + kappa * R) with R the regularisation image."""
    w = np.sum(np.abs(np.asarray(csm, np.complex128)) ** 2, axis=0)
    if reg_image is not None:
        w = w + kappa * np.asarray(reg_image, np.float64)
    return 1.0 / np.sqrt(w)


def cg_solve_refined(op, d: np.ndarray, iterations: int, refinements: int):
    """Outer iterative refinement around cg_solve (new surface, no reference
    counterpart): x_0 = 0; for k = 0..R-1, solve the normal equations for the
    residual right-hand side b - A x_k with `iterations` CG steps from zero
    and add the correction.  complex128 throughout."""
    rhs0 = op.mult_MH(d)
    x = np.zeros_like(rhs0)

    class _Res:
        def __init__(self, rhs):
            self.rhs = rhs

        def mult_MH(self, _):
            return self.rhs

        def mult_MH_M(self, v):
            return op.mult_MH_M(v)

    for k in range(refinements):
        rhs = rhs0 if k == 0 else rhs0 - op.mult_MH_M(x)
        x = x + cg_solve(_Res(rhs), None, iterations=iterations, tc_tolerance=0.0)
    return x


def cg_solve(op, d: np.ndarray, iterations: int = 10, tc_tolerance: float = 1e-3,
             x0=None, precond_weights=None, history=None, regularization=None):
    """cgSolver::solve (cgSolver.h:105-390), complex128 throughout.

    Unpreconditioned: rq = ||r||^2, alpha = rq / <p, q> (complex, Cdotc),
    p <- p * (rq'/rq) + r.  Stops when rq/rq0 < tc_tolerance
    (relativeResidualTCB).  ``regularization``: list of (weight, R) with R
    a real diagonal (the image regulariser's image, or 1 for the identity);
    the operator is E^H E + sum weight * R^2 (cgSolver.h:355-390)."""
    if regularization:
        base = op

        class _Reg:
            def mult_MH(self, y):
                return base.mult_MH(y)

            def mult_MH_M(self, x):
                out = base.mult_MH_M(x)
                for w, R in regularization:
                    R = np.asarray(R, np.float64)
                    out = out + w * (x * R * R)
                return out
        op = _Reg()
    rhs = op.mult_MH(d)
    if iterations == 0:
        return rhs
    vdot = lambda a, b: np.vdot(a.ravel(), b.ravel())
    x = np.zeros_like(rhs)
    r = rhs.copy()
    p = r.copy()
    P = None if precond_weights is None else np.asarray(precond_weights)
    if P is not None:
        p = p * P * P
    rq0 = float(np.real(vdot(r, p)))
    if x0 is not None:
        x = np.asarray(x0, np.complex128).copy()
        r = r - op.mult_MH_M(x)
        p = r.copy()
        if P is not None:
            p = p * P * P
    rq = float(np.real(vdot(r, p)))
    for it in range(iterations):
        q = op.mult_MH_M(p)
        alpha = rq / vdot(p, q)
        x = x + alpha * p
        r = r - alpha * q
        if P is not None:
            q = r * P * P
            tmp_rq = float(np.real(vdot(r, q)))
            p = p * (tmp_rq / rq) + q
        else:
            tmp_rq = float(np.real(vdot(r, r)))
            p = p * (tmp_rq / rq) + r
        rq = tmp_rq
        if history is not None:
            history.append(rq / rq0)
        if rq / rq0 < tc_tolerance:
            break
    return x


# ------------------------------------------------------- radial utilities ---

_PI32 = np.float32(np.pi)


def _fma32(a, b, c):
    """float32 a * b + c with one rounding (the product of two floats is
    exact in double; the sum is rounded to double, then to float)."""
    return (np.asarray(a, np.float64) * np.float64(b) + np.asarray(c, np.float64)).astype(np.float32)


def _gr_step(mode: int) -> np.float32:
    """get_angle_step_GR<float, mode> (radial_utilities.cu:18-23)."""
    s5 = np.sqrt(np.float32(5.0))
    if mode == 0:
        return np.float32(np.float32(_PI32 * (np.float32(3.0) - s5)) * np.float32(0.5))
    return np.float32(_PI32 / np.float32((s5 + np.float32(1.0)) * np.float32(0.5)))


def _pos(S: int, cos_a, sin_a):
    s = np.arange(S, dtype=np.float32)
    Sf = np.float32(S)
    b = np.float32(Sf * np.float32(0.5))
    d = (s - b).astype(np.float32)
    x = (d[None, :] * cos_a[:, None]).astype(np.float32) / Sf
    y = (d[None, :] * sin_a[:, None]).astype(np.float32) / Sf
    return np.stack([x.astype(np.float32), y.astype(np.float32)], -1)


def radial_trajectory_golden_ratio_2d(S: int, P: int, F: int = 1, profile_offset: int = 0, mode: int = 1):
    """compute_radial_trajectory_golden_ratio_2d (radial_utilities.cu:25-87):
    [F, P*S, 2] float32; profile p over all frames at
    (p + offset) * step + pi."""
    prof = np.arange(P * F, dtype=np.float32)
    # (p + offset) * step + pi as one fused multiply-add (nvcc contracts it)
    ang = _fma32((prof + np.float32(profile_offset)).astype(np.float32), _gr_step(mode), _PI32)
    pos = _pos(S, np.cos(ang).astype(np.float32), np.sin(ang).astype(np.float32))
    return pos.reshape(F, P * S, 2)


def radial_trajectory_fixed_angle_2d(S: int, P: int, F: int = 1, angular_offset: float = 0.0):
    """compute_radial_trajectory_fixed_angle_2d (radial_utilities.cu:143-199):
    profile l of frame f at (l + f/F)/P * pi + angular_offset + pi."""
    inv_p, inv_f = np.float32(1.0) / np.float32(P), np.float32(1.0) / np.float32(F)
    f = np.repeat(np.arange(F, dtype=np.float32), P)
    l = np.tile(np.arange(P, dtype=np.float32), F)
    a = (_fma32(f, inv_f, l) * inv_p).astype(np.float32)
    ang = (_fma32(a, _PI32, np.float32(angular_offset)) + _PI32).astype(np.float32)
    pos = _pos(S, np.cos(ang).astype(np.float32), np.sin(ang).astype(np.float32))
    return pos.reshape(F, P * S, 2)


def radial_trajectory_variable_angle_2d(angles, S: int, P: int, F: int):
    """compute_radial_trajectory_variable_angle_2d (radial_utilities.cu:89-140):
    every profile of frame f at angles[f]."""
    ang = np.repeat(np.asarray(angles, np.float32)[:F], P)
    pos = _pos(S, np.cos(ang).astype(np.float32), np.sin(ang).astype(np.float32))
    return pos.reshape(F, P * S, 2)


def radial_dcw_2d(S: int, P: int, alpha: float, ovs: float, profile_offset: int = 0, golden: bool = True,
                  mode: int = 1) -> np.ndarray:
    """compute_radial_dcw_2d (radial_utilities.cu:200-396): the area of the
    polygon through the midpoints towards the sample's two neighbours on its
    profile and, on either side of the profile, the nearest sample of any
    other profile (either half-line) with its two profile neighbours; the
    centre sample gets pi (alpha ovs / 2)^2 / P.  Profile angles without + pi.
    Returns [P*S] float32 (one frame)."""
    f32 = np.float32
    alpha, ovs = f32(alpha), f32(ovs)
    if golden:
        ang = ((np.arange(P, dtype=f32) + f32(profile_offset)) * _gr_step(mode)).astype(f32)
    else:
        ang = ((np.arange(P, dtype=f32) * (f32(1.0) / f32(P))).astype(f32) * _PI32).astype(f32)
    cs, sn = np.cos(ang).astype(f32), np.sin(ang).astype(f32)
    Sf = f32(S)
    bias = f32(Sf * f32(0.5))
    s = np.arange(S, dtype=f32)
    sc = lambda v: (alpha * (v.astype(f32) * ovs).astype(f32)).astype(f32)
    ctr, ctr_inv = sc(s - bias), sc((Sf - s).astype(f32) - bias)
    prv, prv_inv = sc((s - bias).astype(f32) - f32(1.0)), sc((Sf - (s - f32(1.0))).astype(f32) - bias)
    nxt, nxt_inv = sc((s - bias).astype(f32) + f32(1.0)), sc((Sf - (s + f32(1.0))).astype(f32) - bias)
    out = np.zeros((P, S), f32)
    r = f32(f32(alpha * ovs) * f32(0.5))
    big = np.finfo(np.float32).max
    for p in range(P):
        c0, s0 = cs[p], sn[p]
        pos = np.stack([ctr * c0, ctr * s0], -1).astype(f32)          # [S, 2]
        nrm = np.array([-s0, c0], f32)
        A = np.full((3, S, 2), big, f32)
        B = np.full((3, S, 2), big, f32)
        da = np.full(S, np.inf)
        db = np.full(S, np.inf)
        for i in range(P):
            if i == p:
                continue
            d = np.array([cs[i], sn[i]], f32)
            for c_s, p_s, n_s in ((ctr, prv, nxt), (ctr_inv, prv_inv, nxt_inv)):
                cpos = (c_s[:, None] * d[None]).astype(f32)
                side = ((cpos - pos) * nrm[None]).astype(f32).sum(-1)
                dist = (((cpos - pos).astype(np.float64)) ** 2).sum(-1)
                pa = side > 0
                upd_a = pa & (dist < da)
                upd_b = (~pa) & (dist < db)
                for tgt, upd, dd in ((A, upd_a, da), (B, upd_b, db)):
                    tgt[0][upd] = (p_s[upd, None] * d[None]).astype(f32)
                    tgt[1][upd] = cpos[upd]
                    tgt[2][upd] = (n_s[upd, None] * d[None]).astype(f32)
                    dd[upd] = dist[upd]
        own_p = np.stack([prv * c0, prv * s0], -1).astype(f32)
        own_n = np.stack([nxt * c0, nxt * s0], -1).astype(f32)
        verts = [own_p, A[0], A[1], A[2], own_n, B[2], B[1], B[0]]
        m = [(f32(0.5) * (pos + v).astype(f32)).astype(np.float64) for v in verts]
        area = np.zeros(S)
        for k in range(8):
            u, t = m[k], m[(k + 1) % 8]
            area += u[:, 0] * t[:, 1] - t[:, 0] * u[:, 1]
        w = np.abs(0.5 * area).astype(f32)
        w[S // 2] = f32(f32(r * r) * _PI32) / f32(P)
        out[p] = w
    return out.reshape(-1)


# ------------------------------------------------------- b1 map -------------

def estimate_b1_map(coil_images: np.ndarray, D: int, target_coils: int = -1) -> np.ndarray:
    """estimate_b1_map (b1_map.cu:29-118) in FP64: coil_images [C, *image]
    (x last).  RSS-normalise the first target coils, correlation matrices
    A[a][b] = x_b conj(x_a), 7^D box smoothing with zeros outside the image
    (scaled by 1/7^D), two power iterations t_j = sum_k A[k][j] b_k from
    b = 1, then b_c * exp(-i arg b_0)."""
    x = np.asarray(coil_images, np.complex128)
    C = x.shape[0]
    nt = C if (target_coils <= 0 or target_coils > C) else target_coils
    x = x[:nt]
    x = x / np.sqrt(np.sum(np.abs(x) ** 2, axis=0))[None]
    A = x[None, :] * np.conj(x[:, None])                 # A[a, b] = x_b conj(x_a)
    for ax in range(2, 2 + D):                           # separable 7-box, zero padded
        n = A.shape[ax]
        pad = [(0, 0)] * A.ndim
        pad[ax] = (3, 3)
        P = np.pad(A, pad)
        c = np.cumsum(P, axis=ax)
        c = np.concatenate([np.zeros_like(np.take(c, [0], axis=ax)), c], axis=ax)
        A = np.take(c, np.arange(7, n + 7), axis=ax) - np.take(c, np.arange(0, n), axis=ax)
    A = A / 7.0 ** D
    b = np.ones((nt,) + x.shape[1:], np.complex128)
    for _ in range(2):
        t = np.einsum("kj...,k...->j...", A, b)
        b = t / np.sqrt(np.sum(np.abs(t) ** 2, axis=0))[None]
    return b * np.exp(-1j * np.angle(b[0]))[None]


# ------------------------------------------------------- SENSE buffer -------

class OracleSenseBuffer:
    """cuBuffer / cuSenseBuffer (cuBuffer.cpp:7-166, cuSenseBuffer.cpp:18-35):
    num_cycles + 1 oversampled k-space slots; every frame is gridded (NC2C,
    accumulating) into the current slot; after num_sub_cycles frames the slot
    is added to the running sum and the next slot is subtracted and cleared."""

    def __init__(self, N, mos, W, num_coils, num_cycles, num_sub_cycles):
        self.N, self.mos, self.W = tuple(N), tuple(mos), W
        self.C = num_coils
        self.cycle_length = num_cycles + 1
        self.sub_cycle_length = num_sub_cycles
        self.acc = np.zeros((self.C, 1) + self.mos[::-1], np.complex128)
        self.cyc = np.zeros((self.cycle_length,) + self.acc.shape, np.complex128)
        self.cur_idx = self.cur_sub_idx = 0
        self.acc_empty = True
        self.dcw = None
        self.acc_image = None

    def add_frame_data(self, samples, traj) -> bool:
        plan = OraclePlan(self.N, self.mos, self.W)
        D = len(self.N)
        plan.preprocess(np.asarray(traj, np.float32).reshape(1, -1, D))
        s = np.asarray(samples, np.complex128).reshape(self.C, 1, -1)
        if self.dcw is not None:
            s = s * np.asarray(self.dcw, np.float64).reshape(1, 1, -1)
        self.cyc[self.cur_idx] = plan.convolve_nc2c(s, accumulate_into=self.cyc[self.cur_idx])
        done = False
        if self.cur_sub_idx == self.sub_cycle_length - 1:
            done = True
            self.acc = self.acc + self.cyc[self.cur_idx]
            self.acc_empty = False
            self.cur_idx = (self.cur_idx + 1) % self.cycle_length
            self.acc = self.acc - self.cyc[self.cur_idx]
            self.cyc[self.cur_idx] = 0
        self.cur_sub_idx = (self.cur_sub_idx + 1) % self.sub_cycle_length
        return done

    def get_accumulated_coil_images(self):
        D = len(self.N)
        if self.acc_empty:
            self.acc_image = np.ones((self.C,) + self.N[::-1], np.complex128)
        else:
            plan = OraclePlan(self.N, self.mos, self.W)
            img = plan.deapodize(plan.fft(self.acc, forward=False, do_scale=True))
            self.acc_image = crop(img, self.N, D)[:, 0]
        return self.acc_image

    def get_combined_coil_image(self, csm):
        if self.acc_image is None:
            self.get_accumulated_coil_images()
        return np.sum(np.conj(np.asarray(csm, np.complex128)) * self.acc_image, axis=0)


# ------------------------------------------------- density compensation -----

_JINC_NORM_RADIUS = np.float32(0.96960938)
_JINC_C = [np.float32(c) for c in (0.999923599661866, 0.014023570134078, -2.969947516849635,
                                   0.891173008769047, 2.326043034495162, -1.270644932677047)]


def jinc_weight(ad: np.ndarray, R) -> np.ndarray:
    """JincKernel::get (ConvolutionKernel.hpp:165-170, 349-397) for absolute
    offsets ad [..., D] (float32): 0 if any |u_d| > R; else r = |u| / R,
    0 if r >= 0.96960938, else the degree-5 polynomial clipped at 0."""
    ad = np.asarray(ad, np.float32)
    R = np.float32(R)
    r = np.sqrt(np.sum(ad.astype(np.float64) ** 2, axis=-1)).astype(np.float32) / R
    v = np.full(r.shape, _JINC_C[0], np.float64)
    for k in range(1, 6):
        v = v + np.float64(_JINC_C[k]) * np.power(r.astype(np.float64), k)
    v = np.maximum(v, 0.0)
    return np.where((r >= _JINC_NORM_RADIUS) | np.any(ad > R, axis=-1), 0.0, v)


def estimate_dcw(traj: np.ndarray, matrix_size, os_factor: float, num_iterations: int, kernel_width: float = 5.5,
                 initial_dcw=None) -> np.ndarray:
    """estimate_dcw (SDC.hpp:19-80, cuSDC.cu): w <- w / C2NC(NC2C(w)) with the
    Jinc kernel on a grid of round_up_32(N * os) cells per dimension (periodic),
    sample coordinate s = k mos + mos/2, taps [ceil(s - R), floor(s + R)].
    Sums in FP64."""
    traj = np.asarray(traj, np.float32).reshape(-1, len(matrix_size))
    M, D = traj.shape
    R = np.float32(_JINC_NORM_RADIUS * np.float32(kernel_width))
    pad = 2 * int(np.ceil(R))
    mos = []
    for n in matrix_size:
        m = int(np.float32(n) * np.float32(os_factor))
        mos.append(((m + 31) // 32) * 32)
    s = np.stack([(_fma32(traj[:, d], np.float32(mos[d]), np.float32((mos[d] + pad) >> 1)) -
                   np.float32(pad // 2)).astype(np.float32) for d in range(D)], -1)
    lo = np.ceil(s - R).astype(np.int64)
    K = int(np.floor(2 * R)) + 2
    # all (sample, footprint cell) pairs with their weights and cell indices
    offs = np.stack(np.meshgrid(*[np.arange(K)] * D, indexing="ij"), -1).reshape(-1, D)   # [K^D, D]
    cells = lo[:, None, :] + offs[None]                                                   # [M, K^D, D]
    ad = np.abs(s[:, None, :] - cells.astype(np.float32))
    inside = np.all(cells <= np.floor(s + R).astype(np.int64)[:, None, :], axis=-1)
    w = jinc_weight(ad, R)
    w[~inside] = 0.0
    idx = np.zeros(cells.shape[:2], np.int64)
    for d in range(D - 1, -1, -1):
        idx = idx * mos[d] + np.mod(cells[..., d], mos[d])
    G = int(np.prod(mos))
    dcw = np.ones(M) if initial_dcw is None else np.asarray(initial_dcw, np.float64).copy()
    for _ in range(num_iterations):
        grid = np.bincount(idx.ravel(), weights=(w * dcw[:, None]).ravel(), minlength=G)
        t = np.sum(w * grid[idx], axis=1)
        dcw = np.where(t == 0, 0.0, dcw / np.where(t == 0, 1.0, t))
    return dcw


def sdc_fixed_point_residual(traj, matrix_size, os_factor, kernel_width, dcw) -> float:
    """max_j |C2NC(NC2C(w))_j - 1| over samples with w_j > 0: the fixed point
    the estimate converges to."""
    traj = np.asarray(traj, np.float32).reshape(-1, len(matrix_size))
    t = estimate_dcw(traj, matrix_size, os_factor, 0, kernel_width)   # builds nothing, returns ones
    del t
    M, D = traj.shape
    R = np.float32(_JINC_NORM_RADIUS * np.float32(kernel_width))
    pad = 2 * int(np.ceil(R))
    mos = [(((int(np.float32(n) * np.float32(os_factor))) + 31) // 32) * 32 for n in matrix_size]
    s = np.stack([(_fma32(traj[:, d], np.float32(mos[d]), np.float32((mos[d] + pad) >> 1)) -
                   np.float32(pad // 2)).astype(np.float32) for d in range(D)], -1)
    lo = np.ceil(s - R).astype(np.int64)
    K = int(np.floor(2 * R)) + 2
    offs = np.stack(np.meshgrid(*[np.arange(K)] * D, indexing="ij"), -1).reshape(-1, D)
    cells = lo[:, None, :] + offs[None]
    inside = np.all(cells <= np.floor(s + R).astype(np.int64)[:, None, :], axis=-1)
    w = jinc_weight(np.abs(s[:, None, :] - cells.astype(np.float32)), R)
    w[~inside] = 0.0
    idx = np.zeros(cells.shape[:2], np.int64)
    for d in range(D - 1, -1, -1):
        idx = idx * mos[d] + np.mod(cells[..., d], mos[d])
    dcw = np.asarray(dcw, np.float64)
    grid = np.bincount(idx.ravel(), weights=(w * dcw[:, None]).ravel(), minlength=int(np.prod(mos)))
    t = np.sum(w * grid[idx], axis=1)
    m = dcw > 0
    return float(np.max(np.abs(t[m] - 1.0)))


# ---------------------------------------------------------------- NDFT ------

def ndft_forward(x: np.ndarray, traj: np.ndarray, mos, dcw=None) -> np.ndarray:
    """Direct FP64 NDFT: x [nb, *N[::-1]] -> y [nb, M]; traj [M, D]."""
    traj = np.ascontiguousarray(traj, dtype=np.float64)
    M, D = traj.shape
    N = tuple(int(n) for n in x.shape[-D:][::-1])
    xs = np.ascontiguousarray(x, np.complex128).reshape(-1, int(np.prod(N)))
    nb = xs.shape[0]
    y = np.zeros((nb, M), np.complex128)
    dc = None if dcw is None else np.ascontiguousarray(dcw, np.float64).ravel()
    lib().or_ndft_forward(D, _p(_u64(N)), 1.0 / np.sqrt(float(np.prod(mos))), M, nb,
                          _p(traj), None if dc is None else _p(dc), _p(xs), _p(y))
    return y


def ndft_adjoint(y: np.ndarray, traj: np.ndarray, N, mos, dcw=None) -> np.ndarray:
    """Direct FP64 adjoint NDFT: y [nb, M] -> x [nb, *N[::-1]]."""
    traj = np.ascontiguousarray(traj, dtype=np.float64)
    M, D = traj.shape
    ys = np.ascontiguousarray(y, np.complex128).reshape(-1, M)
    nb = ys.shape[0]
    x = np.zeros((nb,) + tuple(int(n) for n in N[::-1]), np.complex128)
    dc = None if dcw is None else np.ascontiguousarray(dcw, np.float64).ravel()
    lib().or_ndft_adjoint(D, _p(_u64(N)), 1.0 / np.sqrt(float(np.prod(mos))), M, nb,
                          _p(traj), None if dc is None else _p(dc), _p(ys), _p(x))
    return x


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
