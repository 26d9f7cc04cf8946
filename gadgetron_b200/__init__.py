"""gadgetron_b200: B200 (sm_100a) non-Cartesian NUFFT, SENSE and CG-SENSE.

A drop-in for Gadgetron's GPU non-Cartesian reconstruction path
(cuNFFT_plan / cuNonCartesianSenseOperator / cuCgSolver).  All arithmetic
runs in the CUDA library libgadgetron_b200.so behind the C ABI declared in
include/gadgetron_b200.h; the Python modules mirror the reference interface.

The library is loaded on first use of a name that needs it (gb.NFFT,
gb.cuCgSolver, ...), so importing a pure-numpy helper such as
gadgetron_b200.synthetic does not map the CUDA library; a missing library
still raises ImportError at that first use.
"""
import importlib

__version__ = "0.1.0"

_EXPORTS = {
    "GadgetronB200Error": "._lib", "NotPreprocessedError": "._lib", "TrajectoryRangeError": "._lib",
    "lib": "._lib",
    "NFFT": ".nfft", "ConvolutionType": ".nfft", "NFFT_comp_mode": ".nfft", "NFFT_conv_mode": ".nfft",
    "NFFT_fft_mode": ".nfft", "NFFT_prep_mode": ".nfft", "cuNFFT_plan": ".nfft", "FLAG_AUTOTUNE": ".nfft",
    "FLAG_COMPENSATED": ".nfft", "FLAG_REFERENCE_FOLD": ".nfft",
    "cuNonCartesianSenseOperator": ".sense",
    "cuCgSolver": ".solvers",
    "cuCgPreconditioner": ".operators", "cuImageOperator": ".operators", "sense_precond_weights": ".operators",
    "cuSenseBuffer": ".buffers",
}
_SUBMODULES = ("b1map", "radial", "sdc", "synthetic", "autograd")


def __getattr__(name):
    if name in _SUBMODULES:
        mod = importlib.import_module("." + name, __name__)
        globals()[name] = mod
        return mod
    src = _EXPORTS.get(name)
    if src is None:
        raise AttributeError("module 'gadgetron_b200' has no attribute %r" % name)
    val = getattr(importlib.import_module(src, __name__), name)
    globals()[name] = val
    return val


def __dir__():
    return sorted(list(globals()) + list(_EXPORTS) + list(_SUBMODULES))
