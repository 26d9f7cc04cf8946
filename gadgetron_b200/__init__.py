"""gadgetron_b200: B200 (sm_100a) non-Cartesian NUFFT, SENSE and CG-SENSE.

A drop-in for Gadgetron's GPU non-Cartesian reconstruction path
(cuNFFT_plan / cuNonCartesianSenseOperator / cuCgSolver).  All arithmetic
runs in the CUDA library libgadgetron_b200.so behind the C ABI declared in
include/gadgetron_b200.h; the Python modules mirror the reference interface.
"""
from ._lib import GadgetronB200Error, NotPreprocessedError, TrajectoryRangeError, lib  # noqa: F401
from .nfft import (NFFT, ConvolutionType, NFFT_comp_mode, NFFT_conv_mode, NFFT_fft_mode,  # noqa: F401
                   NFFT_prep_mode, cuNFFT_plan, FLAG_AUTOTUNE, FLAG_COMPENSATED)
from .sense import cuNonCartesianSenseOperator  # noqa: F401
from .solvers import cuCgSolver  # noqa: F401
from .operators import cuCgPreconditioner, cuImageOperator, sense_precond_weights  # noqa: F401
from . import b1map, radial, sdc  # noqa: F401
from .buffers import cuSenseBuffer  # noqa: F401

__version__ = "0.1.0"
